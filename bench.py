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
KERNELS_PER_WINDOW = 11 + 1   # re-list: hash, 3-launch cell scan, scatter, walk, 3-launch triple scan, fill,
                              # reverse sort; + the window kernel


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
    """nvidia-smi clocks/throttle reasons sampled every 50 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0:   # sampler running before timing starts
                time.sleep(0.02)
            self.lines.clear()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def workload(dem, precision, rank):
    import dem_b200.workloads as w
    return w.rsa_500k(seed=w.SEED + rank, precision=precision)


def time_windows(torch, eng, stream, K, flush_buf, win, time_kernels=False):
    """Per-window CUDA events on the engine's stream; L2 flush between windows
    outside the events.  Returns total ms.  With time_kernels, the last timed
    window replays the engine's window graph variant that records CUDA events
    around the re-list and each pair / particle launch (captured beforehand)."""
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    with torch.cuda.stream(stream):
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
    total_ms = time_windows(torch, eng, stream, K, flush, win, time_kernels=True)
    torch.cuda.synchronize()
    clk = clocks.stop()
    # dominant kernel duration: CUDA events inside the last timed window's graph
    kt = eng.window_kernel_times()
    sc = eng.scalars()
    max_ms = max_over_ranks(torch, dist, total_ms, dev, ws)
    dem_steps = K * win
    value = whole_job_rate(w.n, dem_steps, ws, max_ms)

    peak, peak_kind = measured_peak()
    bp = BYTES_PER_PARTICLE[args.precision]
    pairs = sc["pairs"]
    # dominant kernel: the window kernel (every step of a window in one launch).
    # Algorithmic bytes per launch: each particle-step and pair-step touches
    # its fields once (B_p, B_pair per particle-step / pair-step).
    win_bytes_kernel = win * (w.n * bp + pairs * BYTES_PER_PAIR)
    if kt["window_kernel_ms"] > 0:
        kname, kbytes, kms = "k_window", win_bytes_kernel, kt["window_kernel_ms"]
    else:   # per-step kernels: the particle kernel per step
        kname, kbytes, kms = "k_particle", w.n * bp, kt["particle_ms"]
    achieved = kbytes / (kms / 1e3) / 1e9 if kms > 0 else None
    window_bytes = win_bytes_kernel + w.n * (24 + 8 + 16 + 4) + pairs * 64
    traffic = profile_traffic(f"{kname}_rsa500k_{args.precision}")

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

    # --- end to end through the public API with host buffers: pinned host
    # state -> dem_upload_state -> K windows with a scalar read-back each
    # (dem_get_scalars, a host sync) -> final dem_download_state to pinned host
    e2e = None
    if not args.skip_e2e:
        hp = torch.from_numpy(w.pos).pin_memory()
        hr = torch.from_numpy(w.rad).pin_memory()
        out = torch.empty(3 * w.n, dtype=torch.float64).pin_memory()
        outd = torch.empty(3 * w.n, dtype=torch.float64).pin_memory()
        outa = torch.empty(3 * w.n, dtype=torch.float64).pin_memory()
        ke = max(10, K // 5)
        rawb = eng.scalars_raw_bytes()
        raws = torch.empty((ke, rawb), dtype=torch.uint8).pin_memory()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        a.record(stream)
        eng.upload(hp.numpy(), hr.numpy())
        # every window's observables go to pinned host memory as it ends
        # (dem_scalars_enqueue: queued copies, no host wait between windows)
        for k in range(ke):
            eng.step(win)
            eng.scalars_enqueue(raws[k].data_ptr())
        pos_o, pdis_o, angv_o = out.numpy(), outd.numpy(), outa.numpy()
        from dem_b200 import _ptr, check, lib
        check(lib().dem_download_state(eng.handle, _ptr(pos_o), _ptr(pdis_o), _ptr(angv_o)), "download")
        b.record(stream)
        stream.synchronize()
        e2e_status = max(eng.scalars_from_raw(raws[k].data_ptr())["status"] for k in range(ke))
        wall = time.perf_counter() - t0
        ev_ms = a.elapsed_time(b)
        e2e_s = max_over_ranks(torch, dist, max(wall, ev_ms / 1e3) * 1e3, dev, ws) / 1e3
        h2d = 3 * w.n * 8 + w.n * 8
        d2h = 9 * w.n * 8 + ke * rawb
        e2e = {"value": whole_job_rate(w.n, ke * win, ws, e2e_s * 1e3), "unit": UNIT, "windows": ke,
               "h2d_bytes_per_step": h2d / ke, "d2h_bytes_per_step": d2h / ke, "status": e2e_status,
               "timing": "host wall clock and CUDA events, larger of the two; every window's observables "
                         "copied to pinned host memory as it ends and reduced on the host before the clock stops"}

    # --- CPU baseline: the FP64 oracle on this host's cores, bounded sample
    cpu = None
    if rank == 0 and ws == 1 and not args.skip_cpu:
        cpu = cpu_baseline(dem, w, args.cpu_steps)
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
                   "ms_per_dem_step": max_ms / dem_steps, "pairs_per_particle": pairs / w.n,
                   "contacts_per_particle": sc["contacts"] / w.n, "packing_fraction": sc["packing_fraction"],
                   "mean_cn": sc["mean_cn"]},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": kbytes,
                     "note": "algorithmic bytes count every particle-step's fields once; the window kernel "
                             "keeps free particles in registers across its steps, so achieved can exceed the "
                             "copy peak while DRAM traffic (traffic) stays far below the algorithmic bytes",
                     "kernel_ms": kt, "kernel_timing": "CUDA events inside the last timed window's graph "
                     "(mean over its 20 steps)", "step_bytes_per_window": window_bytes,
                     "step_achieved_gbs": window_bytes / (max_ms / K / 1e3) / 1e9},
        "clocks": clk,
        "gpu_launches": KERNELS_PER_WINDOW * K,
        "fp64_plain": fp64,
        "pp_mode": ppm,
        "scale_4m": scale,
        "adjoint": adj,
        "e2e": e2e,
        "cpu_baseline": cpu,
    }
    print(json.dumps(line), flush=True)


def adjoint_cost(dem, torch, stream):
    """settle_50k: 50,000 lognormal spheres (40x40x150 mm) pre-settled for
    20,000 steps, then a 2,000-step window, checkpoints every 100: time of
    the reverse sweep (objective + recompute + reverse) against the plain
    forward window, packing-fraction objective."""
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
    e.adjoint(w.steps, 100, dem.OBJ_PACKING)           # warm-up (allocates the tape)
    e.upload(pos, w.rad, pdis, angv)
    r = e.adjoint(w.steps, 100, dem.OBJ_PACKING)
    e.close()
    return {"workload": w.name, "n_particles": w.n, "window_steps": w.steps, "checkpoint_every": 100,
            "objective": "packing fraction", "forward_window_ms": fwd_ms,
            "checkpointed_forward_ms": r["forward_ms"], "reverse_ms": r["adjoint_ms"],
            "adjoint_over_forward": r["adjoint_ms"] / fwd_ms,
            "d_mu": r["d_pp"]["mu"] + r["d_pw"]["mu"], "d_roll_rel": r["d_pp"]["roll_rel"] + r["d_pw"]["roll_rel"]}


def cpu_baseline(dem, w, steps):
    sys.path.insert(0, str(ROOT))
    from oracle import oracle as orc
    threads = orc.num_threads()
    mat = dem.material_array(w.pp, w.pw)
    st = orc.Stepper(w.pos, w.rad, w.world, w.dt, w.skin, w.cell(), w.density, mat,
                     w.precision == dem.PREC_MIXED, w.relist_interval)
    t0 = time.perf_counter()
    st.step(steps)
    dt = time.perf_counter() - t0
    st.close()
    return {"value": w.n * steps / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{steps} DEM steps ({steps // w.relist_interval} re-lists) of {w.name} from its initial "
                      f"state, FP64 oracle, OpenMP {threads} threads"}


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
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--cpu-steps", type=int, default=1000)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-pp", action="store_true")
    ap.add_argument("--skip-adjoint", action="store_true")
    ap.add_argument("--skip-4m", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
