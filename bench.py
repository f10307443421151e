"""Benchmark of the RCD demosaic + NLM denoise path on B200.

One step = one 6000x4000 (24 MP) RGGB 14-bit mosaic (black 512, white 16383,
read noise 6 DN, gain 0.5 e/DN) through u16 -> normalise -> RCD -> NLM
(7x7 patch, 21x21 search, h = 1.5 x noise sigma at mid grey) on each RGB
channel, with the raw already resident in HBM. The working set (48 MB raw,
288 MB demosaiced, 288 MB output) is larger than the 126 MB L2, so no flush is
needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). Under torchrun every rank develops its own
frame (frame-parallel replicas, no collective on the data path); the timed
region is bracketed by barriers and the time is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mpix/s RCD+NLM @24MP: learned vs plain GPU NLM, 1 B200, ≤0.1 dB vs FP64"
W, H = 6000, 4000
BLACK, WHITE = 512, 16383
GAIN, READ_SIGMA = 0.5, 6.0
SEARCH, PATCH = 10, 3
WB = np.array([2.0, 1.0, 1.0 / 0.7], np.float32)
CPU_SAMPLE = (1536, 1024)  # oracle crop (w, h) of the same frame for the CPU baseline


def workload_config(n_gpus: int) -> dict:
    return {
        "workload": "RCD demosaic + per-channel NLM, 6000x4000 RGGB u16 14-bit (black 512, white 16383), "
                    "Poisson-Gaussian noise g=0.5 e/DN sigma_read=6 DN, patch 7x7, search 21x21, "
                    "h=1.5*sigma at mid grey, f32 RGB out",
        "frame": [W, H], "cfa": "RGGB", "bits": 14, "search": SEARCH, "patch": PATCH,
        "frames_per_step_per_gpu": 1, "parallelism": f"frame-parallel x{n_gpus}",
        "l2": "working set 624 MB > 126 MB L2 (no flush)",
    }


def h_param() -> float:
    rng = WHITE - BLACK
    dn = 0.5 * rng
    return 1.5 * float(np.sqrt(dn / GAIN + READ_SIGMA ** 2) / rng)


class Clocks:
    """Samples nvidia-smi during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm),
                "power_w_max": max(power) if power else None}


def cpu_baseline(threads: int | None = None, repeats: int = 3) -> dict:
    """The oracle (a C++ restatement of the reference's CPU path, OpenMP over
    all host threads) on a crop of the same frame; returns Mpix/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dsref
    import darkslide_b200 as ds

    dsref.build()
    if threads:
        dsref.set_threads(threads)
    cw, ch = CPU_SAMPLE
    x0, y0 = (W - cw) // 2 & ~1, (H - ch) // 2 & ~1
    sc = ds.Scene(seed=1, w=W, h=H, pattern=ds.RGGB, black=BLACK, white=WHITE, gain=GAIN, read_sigma=READ_SIGMA)
    raw = sc.render_host(x0, y0, cw, ch)
    white = np.full(3, WHITE, np.float32)
    pat = ds.RGGB.shifted(x0, y0).codes()
    times = []
    nt = dsref.threads()
    for _ in range(repeats):
        t0 = time.perf_counter()
        cfa = dsref.normalize_u16(raw, pat, BLACK, white)
        rgb = dsref.rcd(cfa, pat, WB)
        dsref.clip_plane(cfa)
        dsref.nlm_rgb(rgb, h_param(), SEARCH, PATCH, nthreads=nt)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    return {"value": cw * ch / t / 1e6, "unit": "Mpix/s", "cores": nt, "kind": "port",
            "sample": f"{cw}x{ch} crop of the 6000x4000 frame (normalise+RCD+clip+NLM x3), median of {repeats}, "
                      f"{t:.2f} s each", "seconds": t}


def read_traffic() -> dict:
    """DRAM bytes per launch at this workload, from the committed ncu summary
    (profiles/dram_traffic.txt: `key = bytes` lines)."""
    out = {}
    path = os.path.join(ROOT, "profiles", "dram_traffic.txt")
    if os.path.exists(path):
        for ln in open(path):
            if "=" in ln and not ln.lstrip().startswith("#"):
                k, v = ln.split("=", 1)
                try:
                    out[k.strip()] = float(v.split()[0])
                except (ValueError, IndexError):
                    pass
    return out


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import dsref

    dsref.build()
    times = []
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(repeats=1)
        if i >= args.warmup:
            times.append(r["seconds"])
    t = sum(times) / len(times)
    cw, ch = CPU_SAMPLE
    v = cw * ch / t / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "Mpix/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.gpus),
        "cpu_baseline": {"value": v, "unit": "Mpix/s", "cores": dsref.threads(), "kind": "port",
                         "sample": f"each step: {cw}x{ch} crop of the 6000x4000 frame through the oracle "
                                   "(C++ restatement of the reference CPU path; the Rust reference cannot be built here)"},
        "e2e": {"value": v, "unit": "Mpix/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch

    ws, rank, local = dist_env()
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    import darkslide_b200 as ds
    from darkslide_b200 import _lib

    ctx = ds.Context(dev.index)
    stream = torch.cuda.Stream(dev)
    ctx.set_stream(stream.cuda_stream)
    L = _lib.lib()
    import ctypes

    vp = ctypes.c_void_p
    hp = h_param()
    white = np.full(3, WHITE, np.float32)
    pat = ds.RGGB.codes()

    sc = ds.Scene(seed=1 + rank, w=W, h=H, pattern=ds.RGGB, black=BLACK, white=WHITE, gain=GAIN,
                  read_sigma=READ_SIGMA)
    with torch.cuda.stream(stream):
        raw = sc.render(dev, ctx=ctx)
        out = torch.empty((H, W, 3), dtype=torch.float32, device=dev)
    stream.synchronize()

    def step(flags=_lib.DSGPU_ASYNC, raw_p=None, out_p=None):
        ctx.check(L.dsgpu_develop_u16(ctx.handle, raw_p or vp(raw.data_ptr()), W, H, W, vp(pat.ctypes.data),
                                      float(BLACK), vp(white.ctypes.data), vp(WB.ctypes.data), float(hp), SEARCH,
                                      PATCH, out_p or vp(out.data_ptr()), vp(0), flags), "dsgpu_develop_u16")

    def barrier():
        if ws > 1:
            import torch.distributed as dist

            dist.barrier()

    for _ in range(args.warmup):
        step()
    stream.synchronize()

    # ---- device-resident timed region
    clocks = Clocks(int(os.environ.get("CUDA_VISIBLE_DEVICES", str(dev.index)).split(",")[dev.index])
                    if os.environ.get("CUDA_VISIBLE_DEVICES") else dev.index)
    ctx.profile(True)
    n0 = ctx.launch_count()
    barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize(dev)
    barrier()
    clk = clocks.stop()
    launches = ctx.launch_count() - n0
    ms = e0.elapsed_time(e1)
    nlm_ms, nlm_n = ctx.stage_ms(_lib.DSGPU_STAGE_NLM)
    dem_ms, dem_n = ctx.stage_ms(_lib.DSGPU_STAGE_DEMOSAIC)
    ctx.profile(False)
    t_max = ms
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    ms_step = t_max / args.steps
    value = ws * W * H * args.steps / (t_max * 1e-3) / 1e6

    # ---- end to end through the C ABI with pinned host buffers
    raw_h = torch.empty((H, W), dtype=torch.uint16).pin_memory()
    raw_h.copy_(raw.cpu())
    out_h = torch.empty((H, W, 3), dtype=torch.float32).pin_memory()
    ctx.set_stream(None)
    ctx.profile(True)
    for _ in range(2):
        step(_lib.DSGPU_HOST, vp(raw_h.data_ptr()), vp(out_h.data_ptr()))
    ctx.profile(True)  # discard warm-up marks
    barrier()
    k_e2e = max(2, min(args.steps, 5))
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        step(_lib.DSGPU_HOST, vp(raw_h.data_ptr()), vp(out_h.data_ptr()))
    t_e2e = time.perf_counter() - t0
    copy_ms, _ = ctx.stage_ms(_lib.DSGPU_STAGE_COPY)
    ctx.profile(False)
    if ws > 1:
        import torch.distributed as dist

        t = torch.tensor([t_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_e2e = float(t.item())
    e2e = ws * W * H * k_e2e / t_e2e / 1e6

    if rank == 0:
        fl, ex2, fl2 = ctx.measure_peaks()
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except (OSError, ValueError):
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        hbm_src = "measured" if "hbm_gbs" in peaks else "fallback"
        # NLM: one exp per (pixel, channel, search offset) -- enhance.rs:58
        updates = W * H * 3 * (2 * SEARCH + 1) ** 2
        nlm_launch_ms = nlm_ms / max(nlm_n, 1)
        achieved_ex2 = updates / (nlm_launch_ms * 1e-3) / 1e9
        dem_launch_ms = dem_ms / max(dem_n, 1)
        rcd_bytes = W * H * (2 + 12)  # u16 in, RGB f32 out
        traffic = read_traffic()
        line = {
            "metric": METRIC, "value": value, "unit": "Mpix/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded gradient+edge scene, Poisson-Gaussian noise)",
            "config": workload_config(ws),
            "path": "plain GPU RCD+NLM (the learned path is not built yet)",
            "roofline": {
                "kernel": "nlm_tile_kernel<3>", "bound": "sfu", "achieved": achieved_ex2, "peak": ex2 / 1e9,
                "unit": "Gexp/s", "frac": achieved_ex2 / (ex2 / 1e9),
                "traffic": (traffic or {}).get("nlm_bytes_per_launch"),
                "algorithmic": f"{updates:.4g} exp per launch (W*H*3*(2S+1)^2, one exp per pixel, channel and offset)",
                "peak_source": "ex2.approx throughput microbenchmark on this GPU (dsgpu_measure_peaks)",
                "launch_ms": nlm_launch_ms, "fp32_peak_tflops": fl / 1e12, "fp32x2_peak_tflops": fl2 / 1e12,
            },
            "roofline_hbm": {
                "kernel": "rcd_tile_kernel<SrcU16>", "bound": "hbm", "achieved": rcd_bytes / (dem_launch_ms * 1e-3) / 1e9,
                "peak": hbm_peak, "unit": "GB/s", "frac": rcd_bytes / (dem_launch_ms * 1e-3) / 1e9 / hbm_peak,
                "traffic": (traffic or {}).get("rcd_bytes_per_launch"),
                "algorithmic": "14 B/px (u16 in, 3xf32 out)", "peak_source": f"{hbm_src} (MEASURED_PEAKS.json hbm_gbs)",
                "launch_ms": dem_launch_ms,
            },
            "e2e": {"value": e2e, "unit": "Mpix/s", "h2d_bytes_per_step": W * H * 2,
                    "d2h_bytes_per_step": W * H * 12, "copy_ms_per_step": copy_ms / k_e2e,
                    "api": "dsgpu_develop_u16 with DSGPU_HOST, pinned host buffers"},
            "gpu_launches": launches,
            "clocks": clk,
        }
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = {k: v for k, v in cpu_baseline().items() if k != "seconds"}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
