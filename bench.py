"""Benchmark of the eSRRF hot path on B200: input Mpx.frames/s.

Workload (default "fht512"): 2-D FHT path, 512x512 uint16 frames x 500, magnification 4,
radius 1.5, sensitivity 2, AVG+VAR+TAC2 (+INT) cumulants over 5 blocks of 100 frames, seeded
synthetic blinking-emitter stack on 40 filaments (esrrf.synth).  One step = one pass of the hot
path over the whole 500-frame stack.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--kernel fused|plain]

`value`: frames resident in HBM, results left in HBM.  `e2e`: the same metric through the
public host API (pinned host frames in, host results out, copies inside the timed region).
`--impl reference` times the reference's own kernels (oracle/_ref: liveSRRF_noInterpolation.cl
compiled for the host, all cores) with the Fourier interpolation done by numpy's FFT, on a
bounded sample of the same workload.
Multi-GPU (torchrun): every rank runs the full workload on its own GPU (rolling blocks are
independent; no collective on the data path), value = all ranks' input Mpx.frames / max time.
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
PKG = os.path.join(ROOT, "nanoj-esrrf_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOADS = {
    # name: (synth workload, frames per block, cumulants)
    "fht512": ("fht512", 100),
    "fht64": ("fht64", 100),
}
# Fixed convention for algorithmic FP32 work: 22 ops per evaluated tap
OPS_PER_TAP = 22.0
FP32_PEAK_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 74.4 at the 1965 MHz max clock


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def taps_per_pixel(M, fwhm):
    """Interior tap count of the FHT path (integer offsets inside the disc, zero excluded)."""
    sigma = np.float32(fwhm) / np.float32(2.354)
    tSO = (np.float32(2) * sigma + np.float32(1)) * np.float32(M)
    R = np.float32(M) * (np.float32(int(np.float32(2) * sigma)) + np.float32(1))
    r0, r1 = -int(R), int(R + 1)
    n = 0
    for j in range(r0, r1 + 1):
        for i in range(r0, r1 + 1):
            d = np.sqrt(np.float32(i * i + j * j))
            if d != 0 and d <= tSO:
                n += 1
    return n


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index),
                                      f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits"],
                                     capture_output=True, text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if len(s) > 3 + i and s[3 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, x):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_sample(stack, M, fwhm, S, n_frames=1):
    """Reference kernels (oracle/_ref, all host cores) on `n_frames` frames of one block, the
    Fourier interpolation of those frames by numpy's FFT, both timed."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    raw = np.ascontiguousarray(stack[:n_frames], np.float32)
    t0 = time.perf_counter()
    interp = O.fht_interpolate_fft(raw, M)
    if kind == "reference":
        O.ref_fht_block(interp, M, fwhm, S)
    else:
        O.fht_block(interp, M, fwhm, S)
    dt = time.perf_counter() - t0
    mpxf = raw.shape[0] * raw.shape[1] * raw.shape[2] / 1e6
    cores = os.cpu_count() or 1
    return {"value": mpxf / dt, "unit": "Mpx*frames/s", "cores": cores, "kind": kind,
            "sample": f"{n_frames} frame(s) of {raw.shape[2]}x{raw.shape[1]}, M{M}: numpy-FFT "
                      f"interpolation + {'reference kernels compiled for the host' if kind == 'reference' else 'C restatement'}"
                      f", OpenMP over {cores} threads; {dt:.2f} s"}


def run_reference(args, world, rank):
    if rank != 0:
        return
    from esrrf import synth

    name, nf = WORKLOADS[args.workload]
    wl = synth.WORKLOADS[name]
    stack = synth.make_stack(name, frames=max(2, args.steps + args.warmup))
    M, fwhm, S = wl.magnification, wl.fwhm, wl.sensitivity
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(stack[i:i + 1], M, fwhm, S, 1)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    dt = sum(1.0 / r["value"] for r in vals) * (wl.width * wl.height / 1e6)
    line = {
        "impl": "reference", "metric": "input Mpx*frames/s (eSRRF 2-D FHT path)", "value": v,
        "unit": "Mpx*frames/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * dt / max(1, len(vals)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 512x512x500 uint16, M4, radius 1.5, S2, "
                               "AVG+VAR+TAC2, blocks of 100 (bounded sample: 1 frame per step)"},
        "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "Mpx*frames/s"},
        "e2e": {"value": v, "unit": "Mpx*frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def read_traffic_summary(kernel):
    """DRAM bytes per launch of the dominant kernel from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f).get(kernel)
    except (OSError, ValueError):
        return None


def run_ours(args, world, rank, local):
    import ctypes

    import torch

    import esrrf
    from esrrf import synth

    torch.cuda.set_device(local)
    name, nf = WORKLOADS[args.workload]
    wl = synth.WORKLOADS[name]
    stack = synth.make_stack(name, frames=args.frames)
    if args.block:
        nf = args.block
    n, h, w = stack.shape
    M, fwhm, S = wl.magnification, wl.fwhm, wl.sensitivity
    n_blocks = n // nf
    L = esrrf.lib()

    eng = esrrf.LiveSRRF_CL()
    eng.initialise(w, h, M, fwhm, S, nf, nf, chosenDevice=local, kernel=args.kernel,
                   framesPerLaunch=args.frames_per_launch)
    H = eng.handle
    eng.setTiming(True)
    WM, HM = w * M, h * M

    # device-resident input and output
    d_stack = torch.from_numpy(stack.view(np.int16)).to(f"cuda:{local}")
    d_out = torch.empty((n_blocks, 4, HM, WM), dtype=torch.float32, device=f"cuda:{local}")
    frame_bytes = h * w * 2
    launches = [0]
    rgc_ms = [0.0]
    rgc_n = [0]

    def step_device():
        base = d_stack.data_ptr()
        for b in range(n_blocks):
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            esrrf._lib.check(H, L.esrrf_calculate_srrf_u16_device(
                H, ctypes.c_void_p(base + b * nf * frame_bytes), nf))
            _, r_ms, nl = eng.lastTiming()
            launches[0] += nl + 1
            rgc_ms[0] += r_ms
            esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(d_out[b].data_ptr())))

    # pinned host input and output for the end-to-end leg
    h_stack = torch.from_numpy(stack.view(np.int16)).pin_memory()
    h_out = torch.empty((n_blocks, 4, HM, WM), dtype=torch.float32).pin_memory()

    def step_e2e():
        base = h_stack.data_ptr()
        for b in range(n_blocks):
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            esrrf._lib.check(H, L.esrrf_calculate_srrf_u16(
                H, ctypes.c_void_p(base + b * nf * frame_bytes), nf))
            esrrf._lib.check(H, L.esrrf_read_srrf(H, ctypes.c_void_p(h_out[b].data_ptr())))

    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        step_device()
    launches[0] = 0
    rgc_ms[0] = 0.0
    barrier(world)
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        ev0.record(stream)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            step_device()
        ev1.record(stream)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    barrier(world)
    # the engine's calls return only after their own stream drained, so the events on the
    # current stream bracket all of the device work
    dev_s = ev0.elapsed_time(ev1) / 1000.0
    t_step = max_over_ranks(world, dev_s / args.steps)
    gpu_launches = launches[0]
    rgc_total_ms = rgc_ms[0]

    # end-to-end through the host API
    for _ in range(max(1, args.warmup // 2)):
        step_e2e()
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    torch.cuda.synchronize()
    e2e_step = max_over_ranks(world, (time.perf_counter() - t0) / args.steps)
    eng.release()

    if rank != 0:
        return
    mpxf = n * h * w / 1e6
    value = world * mpxf / t_step
    e2e_value = world * mpxf / e2e_step

    # roofline of the dominant kernel (fused RGC), per launch
    F = args.frames_per_launch or 8
    launches_rgc = args.steps * n_blocks * ((nf + F - 1) // F)
    avg_launch_s = (rgc_total_ms / 1000.0) / max(1, launches_rgc)
    taps = taps_per_pixel(M, fwhm)
    peaks, peak_src = load_peaks()
    # compulsory HBM bytes of the path per input pixel-frame: raw uint16 in, plus the four
    # float outputs of each block amortised over its frames
    bytes_per_unit = 2.0 + 4 * 4 * M * M / nf
    alg_bytes_launch = F * h * w * bytes_per_unit
    achieved_gbs = alg_bytes_launch / avg_launch_s / 1e9
    ops_launch = F * WM * HM * taps * OPS_PER_TAP
    achieved_tflops = ops_launch / avg_launch_s / 1e12
    cpu = cpu_reference_sample(stack, M, fwhm, S, 1) if not args.no_cpu_baseline else None
    traffic = read_traffic_summary(f"rgc_{args.kernel}_{args.workload}")
    line = {
        "metric": "input Mpx*frames/s (eSRRF 2-D FHT path)",
        "value": value, "unit": "Mpx*frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {w}x{h}x{n} uint16, M{M}, radius {fwhm}, S{S}, "
                               f"AVG+VAR+TAC2+INT, blocks of {nf}", "kernel": args.kernel,
                   "frames_per_launch": F, "l2": "inputs (262 MB) larger than L2",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "Mpx*frames/s", "h2d_bytes_per_step": int(stack.nbytes),
                "d2h_bytes_per_step": int(h_out.numel() * 4)},
        "gpu_launches": gpu_launches,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved_gbs / peaks["hbm_gbs"],
                     "traffic": traffic, "peak_source": peak_src,
                     "kernel": f"fht_rgc_{args.kernel}", "avg_launch_ms": avg_launch_s * 1e3,
                     "alg_bytes_per_launch": alg_bytes_launch},
        "roofline_fp32": {"achieved": achieved_tflops, "peak": FP32_PEAK_NOMINAL_TFLOPS,
                          "unit": "TFLOP/s", "frac": achieved_tflops / FP32_PEAK_NOMINAL_TFLOPS,
                          "ops_per_launch": ops_launch, "taps_per_pixel": taps,
                          "convention": "22 FP32 ops per evaluated tap; nominal peak at 1965 MHz"},
        "clocks": clk.summary(),
        "cpu_baseline": cpu,
        "wall_s_timed": wall,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fht512", choices=sorted(WORKLOADS))
    ap.add_argument("--kernel", default="fused", choices=["fused", "plain"])
    ap.add_argument("--frames-per-launch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--frames", type=int, default=None,
                    help="shorter stack (profiling runs); default: the workload's length")
    ap.add_argument("--block", type=int, default=0, help="frames per block override")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
