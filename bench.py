#!/usr/bin/env python3
"""Benchmark of the B200 DEM packing step: particle-steps/s on the
500,000-sphere lognormal random-sequential-addition workload (100x100x400 mm
box, dt = 5e-7 s, re-list every 20 steps), mixed precision (FP32
list/forces/accumulation, FP64 positions/velocities/tangential history).

One bench step = one re-list window: the list build plus 20 DEM time steps,
replayed as one CUDA graph.  The default K = 500 windows is the workload's
full 10,000 steps from its initial state.  L2 is flushed (256 MiB write)
between bench steps, outside the timed events; within a window the state
stays as hot as it is in a real run.

Besides the headline the JSON line carries: the FP64 plain form and the
particle-parallel force mode on the same workload; the same 500,000 spheres
as a settled bed (every sphere bound, ~3 contacts per sphere: the contact
path under load) with its window kernel's HBM roofline; the
4,000,000-sphere bidisperse workload;
the adjoint window's cost; the end-to-end figure through the public API with
host buffers; and the FP64 oracle on the host cores, whose sample also gives
the mixed form's error against it.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (under torchrun): independent replicas, one per GPU (the step has no
data-path exchange); time = max over ranks; value = all ranks' work / time.
--impl reference: the CPU restatement of the reference step (the reference
itself does not build: its force laws, four kernels and SDK sort/scan are not
in its repository) on the host cores, one DEM step per bench step.
"""
import argparse
import json
import math
import os
import pathlib
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "discrete-element-method-for-packing-cuda-c-code_b200"
BYTES_PER_PARTICLE = {"mixed": 172, "fp64": 200}   # per particle-step, all fields touched once
BYTES_PER_PAIR = 56                                 # ids 8 + FP64 history r+w 48, per pair-step
METRIC = "particle-steps/s @500K spheres"
UNIT = "particle-steps/s"
def launches_per_window(work):
    """Kernels a window graph launches when its outer candidate list stays
    valid (a rebuild adds the 10 launches of the conditional node's body):
    the outer check, the candidate pass with its scans, the fill, the reverse
    rows, and with cluster batches the component pass; then the window
    kernel, which with cluster batches exits unless a batch is too large, the
    batches and the free particles."""
    batching = work.get("batched", -1) >= 0
    relist = 4 + (1 if batching else 0)
    return relist + (3 if batching else 1)


def load_pkg():
    import importlib.util
    if "dem_b200" in sys.modules:
        return sys.modules["dem_b200"]
    spec = importlib.util.spec_from_file_location("dem_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dem_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def max_over_ranks(torch, dist, ms, device, ws):
    """The job's time: the largest per-rank device time (every rank's timed
    region ends at a barrier first)."""
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    if ws > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(n_per_rank, dem_steps, ws, max_ms):
    """Particle-steps/s of all replicas together (weak scaling: each rank
    steps its own n_per_rank particles)."""
    return n_per_rank * dem_steps * ws / (max_ms / 1e3)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def profile_traffic(name):
    """dram bytes per launch from a committed ncu summary (profiles/<name>.md)."""
    p = ROOT / "profiles" / f"{name}.md"
    if not p.exists():
        return None
    m = re.search(r"dram_bytes_per_launch_full_size:\s*([0-9.eE+]+)", p.read_text())
    return float(m.group(1)) if m else None


class ClockSampler:
    """SM clocks and clock-event (throttle) reasons of one GPU, polled through
    NVML every ~1 ms by a background thread while running, so that a timed
    region of a few milliseconds still holds samples; nvidia-smi at 50 ms
    when NVML is unavailable.  Reads settings only."""

    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.samples = []        # (mhz, reasons bitmask)
        self.smax = None
        self.source = None
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self.samples = []
        self._stop.clear()
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            self.source = "nvml, ~1 ms polling"

            def poll():
                while not self._stop.is_set():
                    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                    rs = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((float(mhz), int(rs)))
                    time.sleep(0.001)
            self._t = threading.Thread(target=poll, daemon=True)
            self._t.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 2.0:   # polling before the timed region starts
                time.sleep(0.001)
        except Exception:
            self._t = None
            self._start_smi()

    def _start_smi(self):
        fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={fields}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.source = "nvidia-smi, 50 ms"

            def read():
                for ln in self.proc.stdout:
                    parts = [x.strip() for x in ln.split(",")]
                    try:
                        self.smax = float(parts[1])
                        bits = 0
                        for (nm, b), v in zip(self.REASONS, parts[2:6]):
                            if v.lower().startswith("active"):
                                bits |= b
                        self.samples.append((float(parts[0]), bits))
                    except (ValueError, IndexError):
                        continue
            self._t = threading.Thread(target=read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def stop(self):
        self._stop.set()
        if getattr(self, "proc", None) is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        if self._t is not None:
            self._t.join(timeout=2.0)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": [], "samples": 0, "source": self.source}
        mhz = [m for m, _ in self.samples]
        bits = 0
        for _, b in self.samples:
            bits |= b
        return {"sm_mhz": statistics.median(mhz), "sm_min_mhz": min(mhz), "sm_max_mhz": self.smax,
                "reasons": [nm for nm, b in self.REASONS if bits & b], "samples": len(mhz), "source": self.source}


def workload(dem, precision, rank):
    import dem_b200.workloads as w
    return w.rsa_500k(seed=w.SEED + rank, precision=precision)


def time_windows(torch, eng, stream, K, flush_buf, win, time_kernels=False, label="windows"):
    """Per-window CUDA events on the engine's stream; L2 flush between windows
    outside the events.  Returns total ms.  With time_kernels, the last timed
    window replays the engine's window graph variant that records CUDA events
    around the re-list and the window kernel (captured beforehand).  The
    windows run inside the NVTX range `label` (a profiler can select them:
    ncu --nvtx --nvtx-include "<label>/")."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with torch.cuda.stream(stream), torch.cuda.nvtx.range(label):
        for k in range(K):
            flush_buf.zero_()
            if time_kernels and k == K - 1:
                eng.set_window_timing(True)
            evs[k][0].record(stream)
            eng.step(win)
            evs[k][1].record(stream)
            if time_kernels and k == K - 1:
                eng.set_window_timing(False)
    stream.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


def window_bytes(n, work, win, bp, ncells):
    """Algorithmic bytes of one window (the byte model of the scope table:
    every field of a particle touched once per step it is stepped, B_p per
    particle-step, 56 B per pair-step), split into the window kernel's and the
    re-list's.  A bound particle (a listed pair or a wall candidacy) is
    stepped with the pair phase every step: win x B_p.  A free particle meets
    nothing before the next re-list, so the window kernel reads and writes
    its fields once and runs its steps in registers: B_p per window.  The
    re-list: N (24 pos + 8 key/val + 16 sort + 4 cell start) + 8 C + 64 P
    (the new list's ids and history written, the old list's read)."""
    nb, P = work["bound"], work["pairs"]
    kernel = win * (nb * bp + P * BYTES_PER_PAIR) + (n - nb) * bp
    relist = n * (24 + 8 + 16 + 4) + 8 * ncells + 64 * P
    return kernel, relist


def roofline(kname, kbytes, kms, peak, peak_kind, workload, traffic=None, note=None):
    achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
    r = {"bound": "hbm", "kernel": kname, "workload": workload, "achieved": achieved, "peak": peak, "unit": "GB/s",
         "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind, "traffic": traffic,
         "algorithmic_bytes_per_launch": kbytes, "kernel_ms": kms}
    if note:
        r["note"] = note
    return r


def run_ours(args):
    import torch
    import torch.distributed as dist
    dem = load_pkg()
    ws, rank, local = dist_env()
    if ws > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    dev = torch.device("cuda", local)
    precision = dem.PREC_MIXED if args.precision == "mixed" else dem.PREC_FP64
    w = workload(dem, precision, rank)
    win = w.relist_interval
    K, W = args.steps, args.warmup
    stream = torch.cuda.Stream(device=dev)
    eng = dem.Engine(**w.engine_kwargs())
    eng.set_stream(stream.cuda_stream)
    eng.set_material(w.pp, w.pw)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)   # > 126 MB L2

    # warm-up from the initial state, then restart from it for the timed run
    eng.upload(w.pos, w.rad)
    for _ in range(W):
        eng.step(win)
    eng.set_window_timing(True)   # capture the timing variant of both list buffers' window graphs
    eng.step(2 * win)
    eng.set_window_timing(False)
    eng.scalars()
    eng.upload(w.pos, w.rad)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    torch.cuda.synchronize()
    total_ms = time_windows(torch, eng, stream, K, flush, win, time_kernels=True, label="headline")
    torch.cuda.synchronize()
    clk = clocks.stop()
    # dominant kernel duration: CUDA events inside the last timed window's graph
    kt = eng.window_kernel_times()
    work = eng.window_work()
    sc = eng.scalars()
    max_ms = max_over_ranks(torch, dist, total_ms, dev, ws)
    dem_steps = K * win
    value = whole_job_rate(w.n, dem_steps, ws, max_ms)
    ncells = eng.grid_info()[2]

    peak, peak_kind = measured_peak()
    bp = BYTES_PER_PARTICLE[args.precision]
    kbytes, rbytes = window_bytes(w.n, work, win, bp, ncells)
    note = ("free flight: ~10 % of the spheres are bound (a listed pair or a wall), the rest step in registers; "
            "latency-bound (grid barriers, dependent loads)")
    if kt["window_kernel_ms"] > 0 and work.get("batched") == 1:
        # the batched window's time is k_batch's (the free spheres' kernel runs
        # beside the re-list, from its candidate pass on): its bytes are the
        # bound spheres' and the pairs', every step
        kname, kms = "k_batch", kt["window_kernel_ms"]
        kbytes = win * (work["bound"] * bp + work["pairs"] * BYTES_PER_PAIR)
        note = ("free flight: ~10 % of the spheres are bound (a listed pair or a wall), stepped as cluster batches "
                "(k_batch: one block per batch of whole components, all the window's steps in shared memory, so "
                "its DRAM traffic is far below this per-step byte model); the free ones run in registers "
                "(k_free_run) on the second stream beside the re-list; latency-bound (block barriers)")
    elif kt["window_kernel_ms"] > 0:
        kname, kms = "k_window", kt["window_kernel_ms"]
    else:   # per-step kernels
        kname, kms = "k_pair+k_particle", kt["pair_ms"] + kt["particle_ms"]
    head_roof = roofline(kname, kbytes, kms, peak, peak_kind, w.name,
                         traffic=profile_traffic(f"{kname.replace('+', '_')}_rsa500k_{args.precision}"), note=note)
    head_roof.update({"kernel_timing": "CUDA events inside the last timed window's graph; window_kernel_ms is the "
                                       "window's stepping (one launch of the window kernel, or the batched window: "
                                       "its exiting window kernel and k_batch, joined with k_free_run, which the "
                                       "re-list started) = the window's 20 steps, relist_ms one re-list",
                      "kernel_ms_all": kt, "window_work": work,
                      "step_bytes_per_window": kbytes + rbytes,
                      "step_achieved_gbs": (kbytes + rbytes) / (max_ms / K / 1e3) / 1e9})

    # --- FP64 plain form of the same step (throughput bar for mixed)
    fp64 = None
    if args.precision == "mixed" and not args.skip_fp64:
        e2 = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_FP64})
        e2.set_stream(stream.cuda_stream)
        e2.set_material(w.pp, w.pw)
        e2.upload(w.pos, w.rad)
        with torch.cuda.stream(stream):
            e2.step(3 * win)
        e2.upload(w.pos, w.rad)
        k2 = max(10, K // 5)
        ms2 = time_windows(torch, e2, stream, k2, flush, win)
        s2 = e2.scalars()
        e2.close()
        v2 = w.n * k2 * win / (ms2 / 1e3)
        fp64 = {"value": v2, "unit": UNIT, "windows": k2, "ms_per_window": ms2 / k2,
                "mixed_over_fp64": value / ws / v2, "packing_fraction": s2["packing_fraction"],
                "packing_fraction_mixed": sc["packing_fraction"]}

    # --- particle-parallel (PP) force mode on the same workload
    ppm = None
    if not args.skip_pp:
        e3 = dem.Engine(**{**w.engine_kwargs(), "force_mode": dem.FORCE_PP})
        e3.set_stream(stream.cuda_stream)
        e3.set_material(w.pp, w.pw)
        e3.upload(w.pos, w.rad)
        with torch.cuda.stream(stream):
            e3.step(3 * win)
        e3.upload(w.pos, w.rad)
        k3 = max(10, K // 5)
        ms3 = time_windows(torch, e3, stream, k3, flush, win)
        e3.close()
        ppm = {"value": w.n * k3 * win / (ms3 / 1e3), "unit": UNIT, "windows": k3,
               "pccp_over_pp": (value / ws) / (w.n * k3 * win / (ms3 / 1e3))}

    # --- the same spheres as a settled bed: the contact path under load
    bed = None
    if not args.skip_bed and ws == 1:
        bed = settled_bed(dem, torch, stream, flush, args, peak, peak_kind)

    # --- the 4,000,000-sphere bidisperse workload (mixed): the step at scale
    scale = None
    if not args.skip_4m and args.precision == "mixed" and ws == 1:
        import dem_b200.workloads as wmod
        w4 = wmod.bidisperse_4m()
        e4 = dem.Engine(**w4.engine_kwargs())
        e4.set_stream(stream.cuda_stream)
        e4.set_material(w4.pp, w4.pw)
        e4.upload(w4.pos, w4.rad)
        with torch.cuda.stream(stream):
            e4.step(3 * win)
        e4.upload(w4.pos, w4.rad)
        k4 = max(10, K // 20)
        ms4 = time_windows(torch, e4, stream, k4, flush, win)
        s4 = e4.scalars()
        e4.close()
        scale = {"workload": "bidisperse_4m", "n_particles": w4.n, "value": w4.n * k4 * win / (ms4 / 1e3),
                 "unit": UNIT, "windows": k4, "ms_per_dem_step": ms4 / (k4 * win),
                 "pairs_per_particle": s4["pairs"] / w4.n, "status": s4["status"]}

    # --- adjoint window cost on the pre-settled 50,000-sphere workload
    adj = None
    if not args.skip_adjoint:
        adj = adjoint_cost(dem, torch, stream)

    # --- end to end through the public API with host buffers, the same K
    # windows as the headline: pinned host state -> dem_upload_state -> K
    # windows, each window's observables copied to pinned host memory as it
    # ends (dem_scalars_enqueue) -> dem_download_state of the final state
    e2e = None
    if not args.skip_e2e:
        e2e = end_to_end(dem, torch, dist, eng, w, stream, dev, ws, K, win)

    # --- CPU baseline: the FP64 oracle on this host's cores, bounded sample;
    # the GPU's state after the same steps gives the mixed form's error
    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        cpu = cpu_baseline(dem, w, args.cpu_steps, stream)
    eng.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K, "warmup": W,
        "ms_per_step": max_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic (seeded RSA packing)",
        "config": {"workload": w.name, "n_particles": w.n, "box_mm": list(w.world), "dt_s": 5e-7,
                   "dem_steps_per_bench_step": win, "dem_steps_timed": dem_steps, "precision": args.precision,
                   "relist_interval": win, "skin_d": w.skin, "parallelism": f"replicas x{ws}",
                   "l2": "flushed between bench steps (256 MiB write, outside the timed events)",
                   "ms_per_dem_step": max_ms / dem_steps, "pairs_per_particle": sc["pairs"] / w.n,
                   "contacts_per_particle": sc["contacts"] / w.n, "packing_fraction": sc["packing_fraction"],
                   "mean_cn": sc["mean_cn"]},
        "roofline": head_roof,
        "clocks": clk,
        "gpu_launches": launches_per_window(work) * K,
        "fp64_plain": fp64,
        "pp_mode": ppm,
        "settled_bed": bed,
        "scale_4m": scale,
        "adjoint": adj,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def settled_bed(dem, torch, stream, flush, args, peak, peak_kind):
    """bed_500k: the 500,000 spheres compacted into a bed (velocity
    proportional to height, then gravity) and settled on the GPU, untimed;
    then windows of the production cadence on it, timed: the mixed form (the
    default force mode, with the window kernel's time and roofline), the
    FP64 plain form and the mixed particle-parallel (PP) form, with the bed's
    pairs, contacts and packing fraction."""
    import dem_b200.workloads as wmod
    t0 = time.perf_counter()
    w0 = wmod.bed_500k_initial()
    if args.bed_load:   # a bed settled and saved by an earlier run (--bed-save)
        z = np.load(args.bed_load)
        meta = dict(w0.meta, pdis=z["pdis"], angv=z["angv"], settle_steps=int(z["settle_steps"]),
                    settled={"status": int(z["status"])})
        w = wmod.Workload(w0.name, w0.n, z["pos"], w0.rad, w0.world, w0.dt, w0.steps, 20, w0.skin, w0.precision,
                          w0.pp, w0.pw, meta=meta)
    else:
        w = wmod.dense_bed(dem, w0, w0.meta["compact_steps"] + args.bed_settle_steps, stream=stream.cuda_stream)
        if args.bed_save:
            np.savez(args.bed_save, pos=w.pos, pdis=w.meta["pdis"], angv=w.meta["angv"],
                     settle_steps=w.meta["settle_steps"], status=w.meta["settled"]["status"])
    settle_s = time.perf_counter() - t0
    pdis, angv = w.meta["pdis"], w.meta["angv"]
    win = w.relist_interval
    kb = args.bed_windows
    out = {"workload": w.name, "n_particles": w.n, "box_mm": list(w.world),
           "init": w.meta["init"], "settle_steps": w.meta["settle_steps"], "settle_s": settle_s,
           "settle_status": w.meta["settled"]["status"]}
    for prec, key, fm in ((dem.PREC_MIXED, "mixed", dem.FORCE_PCCP), (dem.PREC_FP64, "fp64", dem.FORCE_PCCP),
                          (dem.PREC_MIXED, "mixed_pp", dem.FORCE_PP)):
        if key not in args.bed_precisions.split(","):
            continue
        e = dem.Engine(**{**w.engine_kwargs(), "precision": prec, "force_mode": fm})
        e.set_stream(stream.cuda_stream)
        e.set_material(w.pp, w.pw)
        e.upload(w.pos, w.rad, pdis, angv)
        with torch.cuda.stream(stream):
            e.step(2 * win)
            e.set_window_timing(True)
            e.step(2 * win)
            e.set_window_timing(False)
        ms = time_windows(torch, e, stream, kb, flush, win, time_kernels=True, label=f"bed {key}")
        kt = e.window_kernel_times()
        work = e.window_work()
        s = e.scalars(raise_on_status=False)
        ncells = e.grid_info()[2]
        e.close()
        bp = BYTES_PER_PARTICLE[key.split("_")[0]]
        kbytes, rbytes = window_bytes(w.n, work, win, bp, ncells)
        r = {"value": w.n * kb * win / (ms / 1e3), "unit": UNIT, "windows": kb, "ms_per_dem_step": ms / (kb * win),
             "pairs_per_particle": s["pairs"] / w.n, "contacts_per_particle": s["contacts"] / w.n,
             "mean_cn": s["mean_cn"], "packing_fraction": s["packing_fraction"], "status": s["status"],
             "window_work": work, "kernel_ms": kt}
        if kt["window_kernel_ms"] > 0 and fm == dem.FORCE_PCCP:
            r["roofline"] = roofline("k_window", kbytes, kt["window_kernel_ms"], peak, peak_kind, w.name,
                                     traffic=profile_traffic(f"k_window_bed500k_{key}"),
                                     note="every sphere bound: B_p x 20 per sphere + 56 B x 20 per pair")
        r["step_achieved_gbs"] = (kbytes + rbytes) / (ms / kb / 1e3) / 1e9
        out[key] = r
    if "mixed" in out and "fp64" in out:
        out["mixed_over_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    if "mixed" in out and "mixed_pp" in out:   # the particle-parallel force mode on the same bed
        out["pp_over_pccp"] = out["mixed_pp"]["value"] / out["mixed"]["value"]
    out["roofline"] = out.get("mixed", {}).get("roofline")
    return out


def end_to_end(dem, torch, dist, eng, w, stream, dev, ws, K, win):
    """K windows end to end through the public API with host buffers (the
    headline's K), timed by the host clock and by CUDA events (the larger
    counts), and the same with every phase bracketed by events."""
    from dem_b200 import _ptr, check, lib
    hp = torch.from_numpy(w.pos).pin_memory()
    hr = torch.from_numpy(w.rad).pin_memory()
    outs = [torch.empty(3 * w.n, dtype=torch.float64).pin_memory() for _ in range(3)]
    rawb = eng.scalars_raw_bytes()
    raws = torch.empty((K, rawb), dtype=torch.uint8).pin_memory()

    def job(phases=None):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ev[0].record(stream)
        eng.upload(hp.numpy(), hr.numpy())
        if phases is not None:
            ev[1].record(stream)
        for k in range(K):
            eng.step(win)
            eng.scalars_enqueue(raws[k].data_ptr())
        if phases is not None:
            ev[2].record(stream)
        check(lib().dem_download_state(eng.handle, _ptr(outs[0].numpy()), _ptr(outs[1].numpy()),
                                       _ptr(outs[2].numpy())), "download")
        ev[3].record(stream)
        stream.synchronize()
        status = max(eng.scalars_from_raw(raws[k].data_ptr())["status"] for k in range(K))
        wall = time.perf_counter() - t0
        if phases is not None:
            phases.update(upload_ms=ev[0].elapsed_time(ev[1]), windows_ms=ev[1].elapsed_time(ev[2]),
                          download_ms=ev[2].elapsed_time(ev[3]))
        return max(wall * 1e3, ev[0].elapsed_time(ev[3])), status

    job()                      # warm: pinned buffers touched, graphs of this context captured
    ms, status = job()
    phases = {}
    job(phases)
    e2e_ms = max_over_ranks(torch, dist, ms, dev, ws)
    h2d = 3 * w.n * 8 + w.n * 8
    d2h = 9 * w.n * 8 + K * rawb
    return {"value": whole_job_rate(w.n, K * win, ws, e2e_ms), "unit": UNIT, "windows": K,
            "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K, "status": status, "ms": e2e_ms,
            "phases_ms": phases,
            "timing": "host wall clock and CUDA events around upload -> K windows -> download, larger of the two; "
                      "every window's observables copied to pinned host memory as it ends and reduced on the host "
                      "before the clock stops; phases_ms from a second job with events between the phases"}


def adjoint_cost(dem, torch, stream):
    """settle_50k: 50,000 lognormal spheres (40x40x150 mm) pre-settled for
    20,000 steps, then a 2,000-step window, checkpoints every 100, potential
    energy objective (whose friction gradients are not zero: the packing
    fraction's max height belongs to a sphere in free fall).  The whole call
    (checkpointed forward + objective + recompute + reverse) and the reverse
    part alone against the plain forward window."""
    import dem_b200.workloads as wm
    w = wm.settle_50k()
    e = dem.Engine(**w.engine_kwargs())
    e.set_stream(stream.cuda_stream)
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    e.step(w.meta["presettle_steps"])
    pos, pdis, angv = e.download()
    e.upload(pos, w.rad, pdis, angv)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    e.step(w.steps)
    b.record(stream)
    stream.synchronize()
    fwd_ms = a.elapsed_time(b)
    e.upload(pos, w.rad, pdis, angv)
    e.adjoint(w.steps, 100, dem.OBJ_POTENTIAL)           # warm-up (allocates the tape)
    e.upload(pos, w.rad, pdis, angv)
    c, d = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c.record(stream)
    r = e.adjoint(w.steps, 100, dem.OBJ_POTENTIAL)
    d.record(stream)
    stream.synchronize()
    call_ms = c.elapsed_time(d)
    e.close()
    return {"workload": w.name, "n_particles": w.n, "window_steps": w.steps, "checkpoint_every": 100,
            "objective": "potential energy", "forward_window_ms": fwd_ms,
            "checkpointed_forward_ms": r["forward_ms"], "reverse_ms": r["adjoint_ms"], "call_ms": call_ms,
            "call_over_forward": call_ms / fwd_ms,
            "forward_plus_reverse_over_forward": (r["forward_ms"] + r["adjoint_ms"]) / fwd_ms,
            "reverse_over_forward": r["adjoint_ms"] / fwd_ms,
            "d_log_mu": r["d_pp"]["mu"] * w.pp["mu"] + r["d_pw"]["mu"] * w.pw["mu"],
            "d_log_roll_rel": r["d_pp"]["roll_rel"] * w.pp["roll_rel"] + r["d_pw"]["roll_rel"] * w.pw["roll_rel"],
            "objective_value": r["value"]}


def cpu_baseline(dem, w, steps, stream):
    """The FP64 oracle (OpenMP, all host threads) on `steps` DEM steps of the
    workload from its initial state; the mixed GPU form's state after the
    same steps against it: packing fraction, mean coordination number and
    per-particle position RMS (the observables of dempacking.cu:766-776)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as orc
    threads = orc.num_threads()
    mat = dem.material_array(w.pp, w.pw)
    t0 = time.perf_counter()
    o = orc.run(w.pos, w.rad, w.world, w.dt, w.skin, w.cell(), w.density, mat, False, steps, w.relist_interval)
    dt = time.perf_counter() - t0
    e = dem.Engine(**{**w.engine_kwargs(), "precision": dem.PREC_MIXED})
    e.set_stream(stream.cuda_stream)
    e.set_material(w.pp, w.pw)
    e.upload(w.pos, w.rad)
    e.step(steps)
    s = e.scalars()
    pos, _, _ = e.download()
    e.close()
    phi_o = float(np.sum(4.0 / 3.0 * np.pi * w.rad ** 3) / (w.world[0] * w.world[1] * o["maxhz"][-1]))
    cn_o = 2.0 * float(o["ncontacts"][-1]) / w.n
    err = {"steps": steps, "packing_fraction_abs": abs(s["packing_fraction"] - phi_o),
           "mean_cn_abs": abs(s["mean_cn"] - cn_o), "position_rms_d": float(np.sqrt(np.mean((pos - o["pos"]) ** 2))),
           "oracle_status": int(o["status"]), "max_contacts_seen": int(np.max(o["ncontacts"]))}
    return {"value": w.n * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} DEM steps ({steps // w.relist_interval} re-lists) of {w.name} from its initial "
                      f"state, FP64 oracle, OpenMP {threads} threads",
            "mixed_error_vs_oracle": err}


def mapped_libraries():
    """This repository's shared libraries mapped into the process."""
    try:
        maps = pathlib.Path("/proc/self/maps").read_text()
    except OSError:
        return None
    names = sorted({ln.split()[-1] for ln in maps.splitlines() if ln.endswith(".so") and str(ROOT) in ln})
    return [str(pathlib.Path(x).relative_to(ROOT)) for x in names]


def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return
    dem = load_pkg()
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as orc
    import dem_b200.workloads as wmod
    precision = dem.PREC_MIXED if args.precision == "mixed" else dem.PREC_FP64
    w = wmod.rsa_500k(precision=precision)
    threads = orc.num_threads()
    mat = dem.material_array(w.pp, w.pw)
    st = orc.Stepper(w.pos, w.rad, w.world, w.dt, w.skin, w.cell(), w.density, mat,
                     precision == dem.PREC_MIXED, w.relist_interval)
    for _ in range(args.warmup):
        st.step(1)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        st.step(1)
    dt = time.perf_counter() - t0
    st.close()
    value = w.n * args.steps / dt
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded RSA packing)",
        "config": {"workload": w.name, "n_particles": w.n, "dem_steps_per_bench_step": 1,
                   "note": "the reference repository does not build (calforceij/calforceiw, neighborarrayD, "
                           "pairlistD, sumallforceiD, outputporositycnD and the SDK sort/scan are absent); this "
                           "is its step restated in FP64 C++/OpenMP (oracle/dem_oracle.cpp)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{args.steps} DEM steps of {w.name} after {args.warmup} warm-up steps"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "libraries_mapped": mapped_libraries(),
    }
    print(json.dumps(line), flush=True)


def run_bed_only(args):
    import torch
    dem = load_pkg()
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    peak, peak_kind = measured_peak()
    print(json.dumps({"settled_bed": settled_bed(dem, torch, stream, flush, args, peak, peak_kind)}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--cpu-steps", type=int, default=1000)
    ap.add_argument("--bed-settle-steps", type=int, default=5000,
                    help="steps of the bed after its 25,000 compaction steps, before its ten quenches")
    ap.add_argument("--bed-windows", type=int, default=10)
    ap.add_argument("--bed-save", default="", help="save the settled bed (npz) for later --bed-load runs")
    ap.add_argument("--bed-load", default="", help="time a bed saved by --bed-save instead of settling one")
    ap.add_argument("--bed-precisions", default="mixed,fp64,mixed_pp",
                    help="bed rows to time (mixed, fp64; mixed_pp: the particle-parallel force mode)")
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-pp", action="store_true")
    ap.add_argument("--skip-bed", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-4m", action="store_true")
    ap.add_argument("--only-bed", action="store_true",
                    help="the settled bed alone (for profiling its windows: NVTX ranges 'bed mixed', 'bed fp64')")
    args = ap.parse_args()
    if args.only_bed:
        run_bed_only(args)
        return
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
