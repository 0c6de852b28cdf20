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
Multi-GPU (torchrun): the blocks of a world-size times longer stack are split across the ranks
by the library's planner (esrrf_sweep_plan: contiguous runs, one per GPU); blocks are independent,
so there is no collective on the data path; value = all ranks' input Mpx.frames / max time (weak
scaling: the per-GPU work is fixed).
`--drift` gives every frame a seeded shift (vibration correction, loadDriftXYGPUbuffer).
The ncu-derived figures (DRAM traffic, warp instructions per frame) are read from profiles/ only
when that summary's `source_sha:` matches the current kernel sources; otherwise they are reported
as unavailable.
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
    # name: (synth workload, frames per block)
    "fht512": ("fht512", 100),   # 2-D FHT path, the headline workload
    "fht64": ("fht64", 100),     # 2-D FHT path, 64x64 M5
    "sweep256": ("sweep256", 0),  # batched parameter sweep (88 combinations, uneven blocks)
    "mfm3d": ("mfm3d", 200),     # 3-D MFM path, 9 planes
    "adjoint256": ("adjoint256", 100),  # differentiable eSRRF: loss + gradients
    "drift512": ("fht512", 100),  # drift estimation per block of the headline stack
    "bic512": ("fht512", 100),    # 2-D bicubic path with MP correction on the headline stack
}
SWEEP_RADII = [0.5 + 0.25 * i for i in range(11)]
SWEEP_SENS = [1, 2, 3, 4]
SWEEP_MAGS = [2, 4]
# blocks of 37, 64, 99 frames tiling the 200-frame stack, plus an overlapping [0, 100)
SWEEP_BLOCKS = [(0, 37), (37, 64), (101, 99), (0, 100)]
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


def bic_taps_per_pixel(M, fwhm):
    """Interior tap count of the 2-D bicubic path, averaged over the M x M sub-pixel phases: the
    offsets of the 2x gradient grid around (xM + 0.5) / M inside the disc, zero excluded
    (liveSRRF.cl:238-401 geometry, FP32 as the kernel evaluates it)."""
    f = np.float32
    gm = 2
    sigma = f(fwhm) / f(2.354)
    radius = f(int(f(gm * 2) * sigma)) / f(gm) + f(1)
    tSO = f(2) * sigma + f(1)
    r0, r1 = -int(f(gm) * radius), int(f(gm) * radius + f(1))
    cell = 64  # any interior cell
    total = 0
    for py in range(M):
        for px in range(M):
            xc = f((cell * M + px + 0.5) / M)
            yc = f((cell * M + py + 0.5) / M)
            kx, ky = int(f(gm) * xc), int(f(gm) * yc)
            for j in range(r0, r1 + 1):
                dy = f(f(ky + j) / f(gm)) - yc
                for i in range(r0, r1 + 1):
                    dx = f(f(kx + i) / f(gm)) - xc
                    d = np.sqrt(f(dx * dx + dy * dy))
                    if d != 0 and d <= tSO:
                        total += 1
    return total / (M * M)


def taps3d_per_voxel(M, fwhm):
    """Interior tap count of the 3-D path averaged over the M^3 sub-pixel phases: lateral offsets on
    the 2x gradient grid, z offsets on whole planes, inside the sphere, zero excluded
    (live3DSRRF.cl:325-498 geometry, FP32 as the kernel evaluates it)."""
    f = np.float32
    sigma = f(fwhm) / f(2.354)
    radius = f(int(f(4) * sigma)) / f(2) + f(1)
    tSO = f(2) * sigma + f(1)
    r0, r1 = -int(f(2) * radius), int(f(2) * radius + f(1))
    k0, k1 = -int(radius), int(radius) + 1
    total = 0
    for pz in range(M):
        zc = f((pz + 0.5) / M)
        for py in range(M):
            yc = f((py + 0.5) / M)
            ky = int(f(2) * yc)
            for px in range(M):
                xc = f((px + 0.5) / M)
                kx = int(f(2) * xc)
                for j in range(r0, r1 + 1):
                    dy = f(f(ky + j) / f(2)) - yc
                    for i in range(r0, r1 + 1):
                        dx = f(f(kx + i) / f(2)) - xc
                        for k in range(k0, k1 + 1):
                            dz = f(f(int(zc)) + f(k)) - zc
                            d = np.sqrt(f(dx * dx + dy * dy + dz * dz))
                            if d != 0 and d <= tSO:
                                total += 1
    return total / (M ** 3)


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
        # the first nvidia-smi call initialises its driver session, which can take seconds and
        # stall CUDA calls meanwhile: let it finish before the timed region starts
        t0 = time.perf_counter()
        while not self.samples and time.perf_counter() - t0 < 15.0:
            time.sleep(0.05)
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
        # NCCL between GPUs; ESRRF_BENCH_BACKEND=gloo runs the barrier and the max over ranks on the
        # host (ranks sharing one GPU for a functional check: no kernel waits on another rank)
        backend = os.environ.get("ESRRF_BENCH_BACKEND", "nccl")
        kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
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

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def cpu_reference_sample(stack, M, fwhm, S, n_frames=1, bic=False):
    """Reference kernels (oracle/_ref, all host cores) on `n_frames` frames of one block: for the
    FHT path after the Fourier interpolation of those frames by numpy's FFT, both timed; for the
    bicubic path on the raw frames with MP correction."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    raw = np.ascontiguousarray(stack[:n_frames], np.float32)
    t0 = time.perf_counter()
    if bic:
        if kind == "reference":
            O.ref_bic_block(raw, M, fwhm, S, mp_correction=True)
        else:
            O.bic_block(raw, M, fwhm, S, mp_correction=True)
    else:
        interp = O.fht_interpolate_fft(raw, M)
        if kind == "reference":
            O.ref_fht_block(interp, M, fwhm, S)
        else:
            O.fht_block(interp, M, fwhm, S)
    dt = time.perf_counter() - t0
    mpxf = raw.shape[0] * raw.shape[1] * raw.shape[2] / 1e6
    cores = os.cpu_count() or 1
    what = "bicubic path with MP correction" if bic else "numpy-FFT interpolation"
    return {"value": mpxf / dt, "unit": "Mpx*frames/s", "cores": cores, "kind": kind,
            "sample": f"{n_frames} frame(s) of {raw.shape[2]}x{raw.shape[1]}, M{M}: {what} + "
                      f"{'reference kernels compiled for the host' if kind == 'reference' else 'C restatement'}"
                      f", OpenMP over {cores} threads; {dt:.2f} s"}


def cpu_3d_sample(planes, M, fwhm, S, theta, shx, shy, n_tp=2):
    """Reference 3-D kernels (oracle/_ref, all host cores) on the first `n_tp` timepoints' planes,
    with MP correction."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    pl = np.ascontiguousarray(planes[:n_tp], np.float32)
    t0 = time.perf_counter()
    if kind == "reference":
        O.ref_3d_block(pl, M, fwhm, S, theta, shx, shy, mp_correction=True)
    else:
        O.block3d(pl, M, fwhm, S, theta, shx, shy, mp_correction=True)
    dt = time.perf_counter() - t0
    n, P, h, w = pl.shape
    cores = os.cpu_count() or 1
    return {"value": n * P * h * w / 1e6 / dt, "unit": "Mpx*frames/s", "cores": cores, "kind": kind,
            "sample": f"{n} timepoint(s) of {P} planes of {w}x{h}, M{M}: "
                      f"{'reference 3-D kernels compiled for the host' if kind == 'reference' else 'C restatement'}"
                      f", OpenMP over {cores} threads; {dt:.2f} s"}


def cpu_sweep_sample(stack):
    """Reference kernels (oracle/_ref, all host cores) of the sweep: per magnification, the Fourier
    interpolation of one frame (numpy FFT) and the RGC block of that frame at the largest radius,
    each timed; the RGC time is scaled to every radius by its tap count and every combination costs
    its blocks' frame evaluations (ParametersSweep_ runs each combination through the engine)."""
    from oracle import oracle as O

    kind = "reference" if O.ref_available() else "port"
    raw = np.ascontiguousarray(stack[:1], np.float32)
    evals = sum(length for _, length in SWEEP_BLOCKS)  # (start, length) pairs
    rmax = max(SWEEP_RADII)
    total = 0.0
    spent = 0.0
    for M in SWEEP_MAGS:
        t0 = time.perf_counter()
        interp = O.fht_interpolate_fft(raw, M)
        t1 = time.perf_counter()
        if kind == "reference":
            O.ref_fht_block(interp, M, rmax, 1)
        else:
            O.fht_block(interp, M, rmax, 1)
        t2 = time.perf_counter()
        spent += t2 - t0
        per_tap = (t2 - t1) / taps_per_pixel(M, rmax)
        for r in SWEEP_RADII:
            total += len(SWEEP_SENS) * evals * ((t1 - t0) + per_tap * taps_per_pixel(M, r))
    combos = len(SWEEP_MAGS) * len(SWEEP_RADII) * len(SWEEP_SENS)
    cores = os.cpu_count() or 1
    return {"value": combos / total, "unit": "combos/s", "cores": cores, "kind": kind,
            "sample": f"1 frame of {raw.shape[2]}x{raw.shape[1]} per magnification {list(SWEEP_MAGS)} at radius "
                      f"{rmax}: numpy-FFT interpolation + "
                      f"{'reference kernels compiled for the host' if kind == 'reference' else 'C restatement'}"
                      f", OpenMP over {cores} threads ({spent:.2f} s), scaled by tap count to the "
                      f"{combos} combinations x {evals} frame evaluations"}


def path_label(workload):
    return "2-D bicubic path" if workload == "bic512" else "2-D FHT path"


def run_reference(args, world, rank):
    if rank != 0:
        return
    from esrrf import synth

    name, nf = WORKLOADS[args.workload]
    wl = synth.WORKLOADS[name]
    if args.workload == "drift512":
        stack = synth.make_stack(name, frames=20)
        vals = [drift_cpu_sample(stack, 20) for _ in range(args.warmup + args.steps)][args.warmup:]
        v = statistics.median([r["value"] for r in vals])
        print(json.dumps({
            "impl": "reference", "metric": "frames/s (drift estimation)", "value": v, "unit": "frames/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * 20 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "drift512: 512x512 uint16 frames against a reference frame "
                                   "(bounded sample: 20 frames per step)"},
            "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "frames/s"},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "adjoint256":
        print(json.dumps({"impl": "reference", "unavailable": "the fidelity loss and its adjoint are a new "
                          "objective with no reference implementation (the reference scores sweeps with "
                          "ErrorMapLiveSRRF on the CPU, not a differentiable loss)"}))
        return
    if args.workload == "sweep256":
        stack = synth.make_stack("sweep256", frames=2)
        vals = [cpu_sweep_sample(stack) for _ in range(args.warmup + args.steps)][args.warmup:]
        v = statistics.median([r["value"] for r in vals])
        print(json.dumps({
            "impl": "reference", "metric": "sweep combos/s (batched, one CUDA graph)", "value": v,
            "unit": "combos/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * len(SWEEP_MAGS) * len(SWEEP_RADII) * len(SWEEP_SENS) / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "sweep256: 256x256x200, 88 combinations, blocks [0,37) [37,101) "
                                   "[101,200) [0,100) (bounded sample, tap-count scaled)"},
            "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "combos/s"},
            "e2e": {"value": v, "unit": "combos/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    if args.workload == "mfm3d":
        planes = synth.make_stack("mfm3d", frames=2 * (args.steps + args.warmup))
        P = planes.shape[1]
        th = np.linspace(-0.5, 0.5, P).astype(np.float32)
        shx = np.linspace(-0.2, 0.2, P).astype(np.float32)
        shy = np.linspace(0.1, -0.1, P).astype(np.float32)
        vals = [cpu_3d_sample(planes[2 * i:2 * i + 2], 3, 1.5, 1, th, shx, shy, 2)
                for i in range(args.warmup + args.steps)][args.warmup:]
        v = statistics.median([r["value"] for r in vals])
        print(json.dumps({
            "impl": "reference", "metric": "input Mpx*frames/s (eSRRF 3-D MFM path)", "value": v,
            "unit": "Mpx*frames/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * 2 * P * planes.shape[2] * planes.shape[3] / 1e6 / v,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"mfm3d: {P} planes of 128x128 x 200 timepoints, M3, radius 1.5, S1, "
                                   "MP correction (bounded sample: 2 timepoints per step)"},
            "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "Mpx*frames/s"},
            "e2e": {"value": v, "unit": "Mpx*frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))
        return
    bic = args.workload == "bic512"
    per = 2 if bic else 1  # frames per sample (the bicubic path's TAC2 divides by n - 1)
    stack = synth.make_stack(name, frames=max(2, per * (args.steps + args.warmup)))
    M, fwhm, S = wl.magnification, wl.fwhm, wl.sensitivity
    vals = []
    for i in range(args.warmup + args.steps):
        r = cpu_reference_sample(stack[per * i:per * (i + 1)], M, fwhm, S, per, bic=bic)
        if i >= args.warmup:
            vals.append(r)
    v = statistics.median([r["value"] for r in vals])
    dt = sum(1.0 / r["value"] for r in vals) * (per * wl.width * wl.height / 1e6)
    line = {
        "impl": "reference", "metric": f"input Mpx*frames/s (eSRRF {path_label(args.workload)})", "value": v,
        "unit": "Mpx*frames/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * dt / max(1, len(vals)), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: 512x512x500 uint16, M4, radius 1.5, S2, "
                               f"{'bicubic interpolation, MP correction, ' if bic else ''}"
                               f"AVG+VAR+TAC2, blocks of 100 (bounded sample: {per} frame(s) per step)"},
        "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "Mpx*frames/s"},
        "e2e": {"value": v, "unit": "Mpx*frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


TRAFFIC_SUMMARIES = {"rgc_fused_fht512": "rgc_fused_fht512.md", "rgc_fused_bic512": "rgc_bic_bic512.md",
                     "rgc_fused_fht512_drift": "rgc_fused_drift_fht512.md"}
# the kernel sources each summary's counts depend on
SUMMARY_SOURCES = {
    "rgc_fused_fht512": ["fht_fused.cuh", "rgc_fht.cu"],
    "rgc_fused_bic512": ["rgc_bic.cu", "device_common.cuh"],
    "rgc_fused_fht512_drift": ["fht_fused.cuh", "rgc_fht_drift.cu"],
}


def _code_only(text):
    """A C++/CUDA source without its comments, trailing blanks and empty lines (what the compiler
    sees; the kernel sources have no '//' or '/*' inside string literals)."""
    import re

    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    lines = (line.split("//", 1)[0].rstrip() for line in text.splitlines())
    return "\n".join(line for line in lines if line)


def source_sha(kernel):
    """sha256 (first 16 hex digits) of the code of the sources a kernel's ncu figures depend on
    (comments and blank lines removed, so that editing a comment keeps a capture current)."""
    import hashlib

    h = hashlib.sha256()
    for name in SUMMARY_SOURCES.get(kernel, []):
        with open(os.path.join(PKG, "csrc", name), encoding="utf-8") as f:
            h.update(_code_only(f.read()).encode())
    return h.hexdigest()[:16]


def summary_stale(kernel):
    """None if the committed ncu summary of `kernel` was taken of the current sources (its
    `source_sha:` line), else why its figures cannot be used."""
    name = TRAFFIC_SUMMARIES.get(kernel)
    if not name:
        return "no ncu summary for this kernel"
    recorded = None
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith("source_sha:"):
                    recorded = line.split(":", 1)[1].strip()
    except OSError:
        return f"profiles/{name} missing"
    if recorded != source_sha(kernel):
        return (f"profiles/{name} was captured from other kernel sources (sha {recorded}, now "
                f"{source_sha(kernel)}): re-capture before quoting its figures")
    return None


def shard_blocks(world, rank, n_blocks, nf):
    """This rank's blocks under torchrun: the library's planner (esrrf_sweep_plan) splits the
    world * n_blocks blocks of a world-size times longer stack into contiguous runs across the
    ranks (one pair, so blocks are the unit); each rank's run is n_blocks long."""
    if world == 1:
        return list(range(n_blocks))
    import esrrf

    nb = world * n_blocks
    _, bd, _ = esrrf.Sweep.plan(64, 64, nb * nf, [4], [1.5], [2], [(b * nf, nf) for b in range(nb)],
                                list(range(world)))
    mine = [b for b in range(nb) if bd[b] == rank]
    if len(mine) != n_blocks:
        raise RuntimeError(f"planner gave rank {rank} {len(mine)} blocks, expected {n_blocks}")
    return mine


def read_traffic_summary(kernel, key="traffic_bytes_per_launch"):
    """A figure of the dominant kernel from the committed ncu summary (its `<key>:` line: DRAM
    bytes per launch, or warp instructions per frame), if any."""
    name = TRAFFIC_SUMMARIES.get(kernel)
    if not name:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            for line in f:
                if line.startswith(key + ":"):
                    return float(line.split(":", 1)[1])
    except (OSError, ValueError):
        return None
    return None


def secondary_metrics(stack, nf, M, fwhm, S, local, value):
    """The other two figures of the headline metric, measured live on this GPU after the headline
    line's timed regions (bounded: about 10 s): the plain per-pixel kernel on one block of the same
    stack (fused vs plain), the batched sweep of the sweep workload (one graph replay, combos/s)
    and the adjoint of the differentiable workload ((loss + gradients - loss) / loss).  Each is
    timed with CUDA events on the current stream; the calls return after their own streams drained."""
    import ctypes

    import torch

    import esrrf
    from esrrf import synth

    L = esrrf.lib()

    def timed(fn, reps):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        ev0.record()
        for _ in range(reps):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / 1000.0 / reps

    out = {}
    # plain kernel, one block of the headline stack
    h, w = stack.shape[1:]
    eng = esrrf.LiveSRRF_CL()
    eng.initialise(w, h, M, fwhm, S, nf, nf, chosenDevice=local, kernel="plain")
    try:
        H = eng.handle
        d_blk = torch.from_numpy(np.ascontiguousarray(stack[:nf]).view(np.int16)).to(f"cuda:{local}")
        d_o = torch.empty((4, h * M, w * M), dtype=torch.float32, device=f"cuda:{local}")

        def block():
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            esrrf._lib.check(H, L.esrrf_calculate_srrf_u16_device(H, ctypes.c_void_p(d_blk.data_ptr()), nf))
            esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(d_o.data_ptr())))

        block()
        t = timed(block, 1)
        plain = nf * h * w / 1e6 / t
        out["plain"] = {"value": plain, "unit": "Mpx*frames/s", "sample": f"one block of {nf} frames",
                        "fused_over_plain": value / plain}
    finally:
        eng.release()
    del d_blk, d_o
    # batched sweep: 88 combinations x 4 uneven blocks of 256x256x200, one captured graph
    sst = synth.make_stack("sweep256")
    n, sh, sw_ = sst.shape
    sw = esrrf.Sweep(sw_, sh, n, SWEEP_MAGS, SWEEP_RADII, SWEEP_SENS, SWEEP_BLOCKS, device=local)
    try:
        d_s = torch.from_numpy(sst.view(np.int16)).to(f"cuda:{local}")
        d_so = torch.empty(sw.total, dtype=torch.float32, device=f"cuda:{local}")

        def sweep():
            esrrf._lib.check(sw.handle, L.esrrf_sweep_run_device(
                sw.handle, ctypes.c_void_p(d_s.data_ptr()), 1, ctypes.c_void_p(d_so.data_ptr())), sweep=True)

        sweep()  # captures the graph
        combos = len(SWEEP_MAGS) * len(SWEEP_RADII) * len(SWEEP_SENS)
        t = timed(sweep, 2)
        out["sweep"] = {"value": combos / t, "unit": "combos/s", "ms_per_run": t * 1e3,
                        "workload": "sweep256: 256x256x200, 88 combinations, blocks [0,37) [37,101) "
                                    "[101,200) [0,100), device-resident"}
    finally:
        sw.release()
    del d_s, d_so
    # adjoint: loss + all gradients against the loss alone, 256x256x100 at M4
    ast = synth.make_stack("adjoint256").astype(np.float32)
    n, ah, aw = ast.shape
    adj = esrrf.Adjoint(aw, ah, n, 4, device=local)
    try:
        d_a = torch.from_numpy(ast).to(f"cuda:{local}")
        x0 = (1.5, 2.0, 1.5)
        adj.loss(d_a, *x0)
        adj.loss_and_grad(d_a, *x0)
        t_f = timed(lambda: adj.loss(d_a, *x0), 3)
        t_fb = timed(lambda: adj.loss_and_grad(d_a, *x0), 3)
        out["adjoint"] = {"value": (t_fb - t_f) / t_f, "unit": "ratio (loss+grad - loss) / loss",
                          "forward_ms": t_f * 1e3, "loss_and_grad_ms": t_fb * 1e3,
                          "workload": "adjoint256: 256x256x100, M4, AVG"}
    finally:
        adj.release()
    return out


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

    bic = args.workload == "bic512"
    # blocks of this rank: the stack stands for this rank's run of blocks of a world-size times
    # longer stack, split by the library's planner (contiguous runs of balanced frame span)
    blocks_here = shard_blocks(world, rank, n_blocks, nf)
    # vibration correction: a seeded per-frame shift for every block (raw pixels, |s| < 1.5)
    shifts = None
    if args.drift:
        rng = np.random.default_rng(4321)
        shifts = rng.uniform(-1.5, 1.5, size=(n_blocks, 2, nf)).astype(np.float32)
    eng = esrrf.LiveSRRF_CL()
    eng.initialise(w, h, M, fwhm, S, nf, nf, chosenDevice=local, kernel=args.kernel,
                   framesPerLaunch=args.frames_per_launch, doFHTinterpolation=not bic,
                   doMPmapCorrection=bic)
    H = eng.handle
    fpl = ctypes.c_int()
    esrrf._lib.check(H, L.esrrf_frames_per_launch(H, ctypes.byref(fpl)))
    F = fpl.value  # frames per fused launch (the engine's choice unless --frames-per-launch)
    eng.setTiming(True)
    WM, HM = w * M, h * M

    # device-resident input and output
    d_stack = torch.from_numpy(stack.view(np.int16)).to(f"cuda:{local}")
    d_out = torch.empty((n_blocks, 4, HM, WM), dtype=torch.float32, device=f"cuda:{local}")
    frame_bytes = h * w * 2
    launches = [0]
    rgc_ms = [0.0]
    rgc_n = [0]

    fp = ctypes.POINTER(ctypes.c_float)

    def set_drift(b):
        if shifts is not None:
            esrrf._lib.check(H, L.esrrf_set_drift(H, shifts[b, 0].ctypes.data_as(fp),
                                                  shifts[b, 1].ctypes.data_as(fp), nf))

    def step_device():
        base = d_stack.data_ptr()
        for b in range(n_blocks):
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            set_drift(b)
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
        # each block's read-back is queued (esrrf_read_srrf_async) and overlaps the next block's
        # upload and kernels, across steps too, as for a continuous stream; finishQueue after the
        # last step waits for every copy
        base = h_stack.data_ptr()
        for b in range(n_blocks):
            esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
            set_drift(b)
            esrrf._lib.check(H, L.esrrf_calculate_srrf_u16(
                H, ctypes.c_void_p(base + b * nf * frame_bytes), nf))
            esrrf._lib.check(H, L.esrrf_read_srrf_async(H, ctypes.c_void_p(h_out[b].data_ptr())))

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
    esrrf._lib.check(H, L.esrrf_finish_queue(H))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        step_e2e()
    esrrf._lib.check(H, L.esrrf_finish_queue(H))  # every step's results are on the host
    torch.cuda.synchronize()
    e2e_step = max_over_ranks(world, (time.perf_counter() - t0) / args.steps)
    eng.release()

    if rank != 0:
        return
    mpxf = n * h * w / 1e6
    value = world * mpxf / t_step
    e2e_value = world * mpxf / e2e_step

    # roofline of the dominant kernel (fused RGC), per launch
    launches_rgc = args.steps * n_blocks * ((nf + F - 1) // F)
    avg_launch_s = (rgc_total_ms / 1000.0) / max(1, launches_rgc)
    taps = bic_taps_per_pixel(M, fwhm) if bic else taps_per_pixel(M, fwhm)
    peaks, peak_src = load_peaks()
    # compulsory HBM bytes of the path per input pixel-frame: raw uint16 in, plus the block's
    # three cumulant outputs (AVG, VAR, TAC2 in float) amortised over its frames -- the fixed
    # convention of the workload table; INT, a by-product, is not counted
    bytes_per_unit = 2.0 + 3 * 4 * M * M / nf
    alg_bytes_launch = F * h * w * bytes_per_unit
    achieved_gbs = alg_bytes_launch / avg_launch_s / 1e9
    ops_launch = F * WM * HM * taps * OPS_PER_TAP
    achieved_tflops = ops_launch / avg_launch_s / 1e12
    cpu = (cpu_reference_sample(stack, M, fwhm, S, 2 if bic else 1, bic=bic)
           if not args.no_cpu_baseline and world == 1 else None)
    # the headline metric's other figures (fused vs plain, sweep combos/s, adjoint / forward), on
    # the full default workload only
    secondary = (secondary_metrics(stack, nf, M, fwhm, S, local, value)
                 if (world == 1 and args.workload == "fht512" and args.kernel == "fused" and not args.drift
                     and args.frames is None and not args.block and not args.no_cpu_baseline) else None)
    summary_key = f"rgc_{args.kernel}_{args.workload}" + ("_drift" if args.drift else "")
    stale = summary_stale(summary_key)
    traffic = None if stale else read_traffic_summary(summary_key)
    # the kernel's real limit is instruction issue: warp instructions per launch (ncu count per
    # frame x frames) over the live launch time, against one warp instruction per cycle per
    # scheduler (148 SMs x 4) at the sampled SM clock
    clocks = clk.summary()
    ipf = None if stale else read_traffic_summary(summary_key, "warp_instructions_per_frame")
    roofline_issue = None
    if stale:
        roofline_issue = {"unavailable": stale}
    elif ipf and avg_launch_s > 0:
        mhz = clocks.get("sm_mhz") or 1965.0
        peak_issue = 148 * 4 * mhz * 1e6
        got = ipf * (nf / ((nf + F - 1) // F)) / avg_launch_s  # mean frames per launch
        roofline_issue = {"achieved": got, "peak": peak_issue, "unit": "warp instructions/s",
                          "frac": got / peak_issue, "instructions_per_frame": ipf,
                          "source": "instructions per frame from the committed ncu summary of this "
                                    "kernel source (sha recorded there), launch time live"}
    line = {
        "metric": f"input Mpx*frames/s (eSRRF {path_label(args.workload)})",
        "value": value, "unit": "Mpx*frames/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_step * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{args.workload}: {w}x{h}x{n} uint16, M{M}, radius {fwhm}, S{S}, "
                               f"{'bicubic interpolation, MP correction, ' if bic else ''}"
                               f"AVG+VAR+TAC2+INT, blocks of {nf}",
                   "kernel": "bicubic" if bic else args.kernel,
                   "frames_per_launch": F,
                   "l2": (f"inputs ({stack.nbytes / 1e6:.0f} MB) larger than L2" if stack.nbytes > 126e6 else
                          f"inputs ({stack.nbytes / 1e6:.1f} MB) fit in L2, not flushed between steps "
                          "(small parity workload; the kernel reads its interpolated frames, "
                          f"{n * WM * HM * 4 / 1e6:.0f} MB, from HBM)"),
                   "drift": ("seeded per-frame shifts, |s| < 1.5 raw px (vibration correction)"
                             if args.drift else "none"),
                   "parallelism": (f"blocks sharded x{world} (esrrf_sweep_plan: contiguous runs of the "
                                   f"{world * n_blocks} blocks of a {world * n}-frame stack; blocks "
                                   f"{blocks_here[0]}..{blocks_here[-1]} here)" if world > 1 else "1 GPU")},
        "e2e": {"value": e2e_value, "unit": "Mpx*frames/s", "h2d_bytes_per_step": int(stack.nbytes),
                "d2h_bytes_per_step": int(h_out.numel() * 4)},
        "gpu_launches": gpu_launches,
        "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved_gbs / peaks["hbm_gbs"],
                     "traffic": traffic, "peak_source": peak_src,
                     "kernel": "bic_rgc" if bic else f"fht_rgc_{args.kernel}",
                     "avg_launch_ms": avg_launch_s * 1e3,
                     "alg_bytes_per_launch": alg_bytes_launch},
        "roofline_fp32": {"achieved": achieved_tflops, "peak": FP32_PEAK_NOMINAL_TFLOPS,
                          "unit": "TFLOP/s", "frac": achieved_tflops / FP32_PEAK_NOMINAL_TFLOPS,
                          "ops_per_launch": ops_launch, "taps_per_pixel": taps,
                          "convention": "22 FP32 ops per evaluated tap; nominal peak at 1965 MHz"},
        "roofline_issue": roofline_issue,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "wall_s_timed": wall,
    }
    if secondary:
        line["secondary"] = secondary
    print(json.dumps(line))


def run_sweep(args, world, rank, local):
    """Batched sweep (one captured graph) against a loop of single-combination plain-kernel
    engine runs, the structure of ParametersSweep_.run; metric combos/s."""
    import ctypes

    import torch

    import esrrf
    from esrrf import synth

    torch.cuda.set_device(local)
    stack = synth.make_stack("sweep256")
    n, h, w = stack.shape
    L = esrrf.lib()
    sw = esrrf.Sweep(w, h, n, SWEEP_MAGS, SWEEP_RADII, SWEEP_SENS, SWEEP_BLOCKS, device=local)
    d_stack = torch.from_numpy(stack.view(np.int16)).to(f"cuda:{local}")
    d_out = torch.empty(sw.total, dtype=torch.float32, device=f"cuda:{local}")
    combos = len(SWEEP_MAGS) * len(SWEEP_RADII) * len(SWEEP_SENS)

    def step():
        esrrf._lib.check(sw.handle, L.esrrf_sweep_run_device(sw.handle, ctypes.c_void_p(d_stack.data_ptr()),
                                                            1, ctypes.c_void_p(d_out.data_ptr())), sweep=True)

    def timed(fn, n):
        # each sweep call returns after its stream drained: events on the current stream bracket it
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(n):
            fn()
        ev1.record()
        torch.cuda.synchronize()
        return ev0.elapsed_time(ev1) / 1000.0 / n

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_local = timed(step, args.steps)
    barrier(world)
    t_step = max_over_ranks(world, t_local)
    launches = sw.launch_count()
    # e2e: host stack in, host results out
    h_stack = torch.from_numpy(stack.view(np.int16)).pin_memory()
    h_out = torch.empty(sw.total, dtype=torch.float32).pin_memory()
    esrrf._lib.check(sw.handle, L.esrrf_sweep_run(sw.handle, ctypes.c_void_p(h_stack.data_ptr()), 1,
                                                  ctypes.c_void_p(h_out.data_ptr())), sweep=True)
    t0 = time.perf_counter()
    esrrf._lib.check(sw.handle, L.esrrf_sweep_run(sw.handle, ctypes.c_void_p(h_stack.data_ptr()), 1,
                                                  ctypes.c_void_p(h_out.data_ptr())), sweep=True)
    e2e = time.perf_counter() - t0

    # SQUIRREL scoring of every reconstruction (AVG, VAR, TAC2 against the block's INT slice),
    # on the sweep's device-resident output, one batched call per magnification
    def squirrel_all():
        fp = ctypes.POINTER(ctypes.c_float)
        n_img, nR, nS, nB = 0, len(SWEEP_RADII), len(SWEEP_SENS), len(SWEEP_BLOCKS)
        for mi, M in enumerate(SWEEP_MAGS):
            P = h * M * w * M
            sro, rfo = [], []
            for ri in range(nR):
                base = sw.offsets[mi * nR + ri]
                for si in range(nS):
                    for bi in range(nB):
                        blk = base + (si * nB + bi) * 4 * P
                        for c in range(3):
                            sro.append(blk + c * P)
                            rfo.append(blk + 3 * P)
            n = len(sro)
            outs = [np.empty(n, np.float32) for _ in range(5)]
            p = esrrf._lib.EsrrfSquirrelParams(w * M, h * M, M, 0, 0.0, 0,
                                               ctypes.c_void_p(torch.cuda.current_stream(local).cuda_stream))
            esrrf._lib.check(None, L.esrrf_squirrel(ctypes.byref(p), n, ctypes.c_void_p(d_out.data_ptr()),
                                                    (ctypes.c_size_t * n)(*sro), (ctypes.c_size_t * n)(*rfo),
                                                    *[o.ctypes.data_as(fp) for o in outs], None), squirrel=True)
            n_img += n
        return n_img

    sq_images, sq_s = 0, None
    if rank == 0:
        step()
        torch.cuda.synchronize()
        squirrel_all()  # warm-up
        t0 = time.perf_counter()
        sq_images = squirrel_all()
        sq_s = time.perf_counter() - t0
        # CPU stand-in: the float64 restatement on two reconstructions (one per magnification)
        from oracle import squirrel_oracle as Q
        flat = d_out.cpu().numpy()
        t0 = time.perf_counter()
        for mi, M in enumerate(SWEEP_MAGS):
            P = h * M * w * M
            base = sw.offsets[mi * len(SWEEP_RADII) + 4]
            img = flat[base:base + 4 * P].reshape(4, h * M, w * M)
            Q.squirrel(img[0], img[3], M)
        sq_cpu_per_image = (time.perf_counter() - t0) / len(SWEEP_MAGS)

    # FRC resolution of every combination and cumulant (264 pairs): the [0,100) and [101,200)
    # blocks stand in for the odd/even reconstructions of the reference's FRC mode (same sizes)
    def frc_all():
        fp = ctypes.POINTER(ctypes.c_float)
        n_pairs, nR, nS, nB = 0, len(SWEEP_RADII), len(SWEEP_SENS), len(SWEEP_BLOCKS)
        for mi, M in enumerate(SWEEP_MAGS):
            P = h * M * w * M
            ao, bo = [], []
            for ri in range(nR):
                base = sw.offsets[mi * nR + ri]
                for si in range(nS):
                    for c in range(3):
                        ao.append(base + (si * nB + 3) * 4 * P + c * P)
                        bo.append(base + (si * nB + 2) * 4 * P + c * P)
            n = len(ao)
            fire = np.empty(n, np.float32)
            p = esrrf._lib.EsrrfFrcParams(w * M, h * M, 1.0 / M,
                                          ctypes.c_void_p(torch.cuda.current_stream(local).cuda_stream))
            esrrf._lib.check(None, L.esrrf_frc(ctypes.byref(p), n, ctypes.c_void_p(d_out.data_ptr()),
                                               (ctypes.c_size_t * n)(*ao), (ctypes.c_size_t * n)(*bo),
                                               fire.ctypes.data_as(fp), None), frc=True)
            n_pairs += n
        return n_pairs

    frc_pairs, frc_s, frc_cpu_per_pair = 0, None, None
    if rank == 0:
        frc_all()  # warm-up
        t0 = time.perf_counter()
        frc_pairs = frc_all()
        frc_s = time.perf_counter() - t0
        from oracle import frc_oracle as FO
        t0 = time.perf_counter()
        for mi, M in enumerate(SWEEP_MAGS):
            P = h * M * w * M
            base = sw.offsets[mi * len(SWEEP_RADII) + 4]
            a = flat[base + 3 * 4 * P:base + 3 * 4 * P + P].reshape(h * M, w * M)
            b = flat[base + 2 * 4 * P:base + 2 * 4 * P + P].reshape(h * M, w * M)
            FO.fire(a, b)
        frc_cpu_per_pair = (time.perf_counter() - t0) / len(SWEEP_MAGS)
    sw.release()

    # the same sweep on the bicubic path (the sweep's "Use FHT interpolation" option off: bicubic
    # RGC with MP correction), into the same output buffer (same layout)
    swb = esrrf.Sweep(w, h, n, SWEEP_MAGS, SWEEP_RADII, SWEEP_SENS, SWEEP_BLOCKS, device=local,
                      interpolation="bicubic")
    assert swb.total == sw.total

    def step_b():
        esrrf._lib.check(swb.handle, L.esrrf_sweep_run_device(swb.handle, ctypes.c_void_p(d_stack.data_ptr()),
                                                             1, ctypes.c_void_p(d_out.data_ptr())), sweep=True)

    for _ in range(max(1, args.warmup)):
        step_b()
    t_bic = timed(step_b, args.steps)
    bic_launches = swb.launch_count()
    swb.release()

    def single_combo_loop(kernel, subset=None):
        """One engine per combination, every block pushed and read back (device frames)."""
        fb = h * w * 2
        t_total = 0.0
        todo = [(M, r, S) for M in SWEEP_MAGS for r in SWEEP_RADII for S in SWEEP_SENS]
        if subset:
            todo = todo[::subset]
        for (M, r, S) in todo:
            eng = esrrf.LiveSRRF_CL()
            out = torch.empty((4, h * M, w * M), dtype=torch.float32, device=f"cuda:{local}")
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for (st, ln) in SWEEP_BLOCKS:
                eng.initialise(w, h, M, r, S, ln, ln, chosenDevice=local, kernel=kernel)
                H = eng.handle
                esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
                esrrf._lib.check(H, L.esrrf_calculate_srrf_u16_device(
                    H, ctypes.c_void_p(d_stack.data_ptr() + st * fb), ln))
                esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(out.data_ptr())))
            torch.cuda.synchronize()
            t_total += time.perf_counter() - t0
            eng.release()
        return t_total * (subset or 1)

    plain_s = single_combo_loop("plain", subset=8) if rank == 0 else 0.0
    fused_s = single_combo_loop("fused", subset=4) if rank == 0 else 0.0
    if rank != 0:
        return
    line = {
        "metric": "sweep combos/s (batched, one CUDA graph)", "value": world * combos / t_step,
        "unit": "combos/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "sweep256: 256x256x200 uint16, radius 0.5..3.0 (11) x S 1..4 x M {2,4} "
                               "= 88 combinations, blocks [0,37) [37,101) [101,200) [0,100)"},
        "plain_loop_combos_s": combos / plain_s, "fused_loop_combos_s": combos / fused_s,
        "speedup_vs_plain_loop": (combos / t_step) / (combos / plain_s),
        "baseline_note": "single-combination loops re-create the engine per block (as "
                         "ParametersSweep_ re-initialises per combination); plain loop timed on "
                         "every 8th combination, fused loop on every 4th, scaled to 88",
        "e2e": {"value": combos / e2e, "unit": "combos/s", "h2d_bytes_per_step": int(stack.nbytes),
                "d2h_bytes_per_step": int(h_out.numel() * 4)},
        "gpu_launches": launches * args.steps, "clocks": clk.summary(),
        "bicubic": {"combos_per_s": combos / t_bic, "ms_per_run": t_bic * 1e3,
                    "launches_per_run": bic_launches,
                    "what": "the same 88 combinations and 4 blocks on the bicubic path with MP "
                            "correction, one CUDA graph"},
        "squirrel": {"images": sq_images, "seconds": sq_s, "images_per_s": sq_images / sq_s,
                     "what": "RSE, RSP (Brent-optimised blur sigma, alpha/beta fit) of every AVG, "
                             "VAR and TAC2 reconstruction against its block's INT slice",
                     "cpu_port_seconds_per_image": sq_cpu_per_image,
                     "cpu_note": "float64 numpy restatement, one image of each magnification; the "
                                 "reference's own ImageJ/commons-math path needs a JVM"},
        "frc": {"pairs": frc_pairs, "seconds": frc_s, "pairs_per_s": frc_pairs / frc_s if frc_s else None,
                "what": "FIRE resolution (1/7 threshold) of AVG, VAR and TAC2 of every combination, "
                        "blocks [0,100) vs [101,200) standing in for the odd/even halves",
                "cpu_port_seconds_per_pair": frc_cpu_per_pair,
                "cpu_note": "float64 numpy restatement (numpy FFT, one thread), one pair per magnification"},
    }
    print(json.dumps(line))


def run_3d(args, world, rank, local):
    """3-D MFM workload: 9 planes of 128x128 (a 384x384 camera frame) x 200 timepoints, M3,
    radius 1.5, S1, AVG+VAR; one block of all timepoints through the engine."""
    import ctypes

    import torch

    import esrrf
    from esrrf import synth

    torch.cuda.set_device(local)
    planes = synth.make_stack("mfm3d", frames=args.frames)
    n, P, h, w = planes.shape
    roi = np.array([4, 0, 1, 2, 3, 5, 6, 7, 8], np.float32)[:P]
    cam = np.zeros((n, 3 * h, 3 * w), np.uint16)
    for z in range(P):
        i, j = int(roi[z]) % 3, int(roi[z]) // 3
        cam[:, j * h:(j + 1) * h, i * w:(i + 1) * w] = planes[:, z]
    calib = {"X-shift (pixels)": np.linspace(-0.2, 0.2, P), "Y-shift (pixels)": np.linspace(0.1, -0.1, P),
             "Theta (degrees)": np.linspace(-0.5, 0.5, P), "Axial positions": np.zeros(P),
             "ROI #": roi, "Intensity scaling": np.ones(P), "Background level (ADC)": np.full(P, 0.0)}
    M, fwhm, S = 3, 1.5, 1
    eng = esrrf.LiveSRRF_CL()
    d_cam = torch.from_numpy(cam.view(np.int16)).to(f"cuda:{local}")
    d_out = torch.empty((4 * P * M, h * M, w * M), dtype=torch.float32, device=f"cuda:{local}")
    L = esrrf.lib()

    def per_launch_form(fpl):
        """Device time (ms) of one step with `fpl` timepoints per launch (1: the plain form, one
        timepoint at a time)."""
        e2 = esrrf.LiveSRRF_CL()
        e2.initialise(3 * w, 3 * h, M, fwhm, S, n, n, chosenDevice=local, doMPmapCorrection=True,
                      calibTable3DSRRF=calib, framesPerLaunch=fpl, kernel=args.kernel)
        try:
            ts = []
            for i in range(3):
                torch.cuda.synchronize()
                a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a0.record()
                esrrf._lib.check(e2.handle, L.esrrf_reset_frame_position(e2.handle))
                esrrf._lib.check(e2.handle, L.esrrf_calculate_srrf_u16_device(
                    e2.handle, ctypes.c_void_p(d_cam.data_ptr()), n))
                esrrf._lib.check(e2.handle, L.esrrf_read_srrf_device(
                    e2.handle, ctypes.c_void_p(d_out.data_ptr())))
                a1.record()
                torch.cuda.synchronize()
                if i > 0:
                    ts.append(a0.elapsed_time(a1))
            return min(ts)
        finally:
            e2.release()

    plain_ms = per_launch_form(1) if world == 1 else None
    eng = esrrf.LiveSRRF_CL()
    eng.initialise(3 * w, 3 * h, M, fwhm, S, n, n, chosenDevice=local, doMPmapCorrection=True,
                   calibTable3DSRRF=calib, framesPerLaunch=args.frames_per_launch, kernel=args.kernel)
    H = eng.handle
    tpl = ctypes.c_int(0)
    esrrf._lib.check(H, L.esrrf_frames_per_launch(H, ctypes.byref(tpl)))  # the engine's choice
    eng.setTiming(True)
    launches = [0]
    rgc_ms = [0.0]

    def step():
        esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
        esrrf._lib.check(H, L.esrrf_calculate_srrf_u16_device(H, ctypes.c_void_p(d_cam.data_ptr()), n))
        _, r_ms, nl = eng.lastTiming()
        launches[0] += nl + 3
        rgc_ms[0] += r_ms
        esrrf._lib.check(H, L.esrrf_read_srrf_device(H, ctypes.c_void_p(d_out.data_ptr())))

    for _ in range(args.warmup):
        step()
    launches[0] = 0
    rgc_ms[0] = 0.0
    barrier(world)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # the engine's calls return only after their own stream drained, so events on the current
        # stream bracket all of the device work
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    t_step = max_over_ranks(world, ev0.elapsed_time(ev1) / 1000.0 / args.steps)
    rgc_timed = [rgc_ms[0]]
    h_cam = torch.from_numpy(cam.view(np.int16)).pin_memory()
    h_out = torch.empty((4 * P * M, h * M, w * M), dtype=torch.float32).pin_memory()
    t0 = time.perf_counter()
    esrrf._lib.check(H, L.esrrf_reset_frame_position(H))
    esrrf._lib.check(H, L.esrrf_calculate_srrf_u16(H, ctypes.c_void_p(h_cam.data_ptr()), n))
    esrrf._lib.check(H, L.esrrf_read_srrf(H, ctypes.c_void_p(h_out.data_ptr())))
    e2e = time.perf_counter() - t0
    eng.release()
    if rank != 0:
        return
    mpxf = n * P * h * w / 1e6
    th = np.asarray(calib["Theta (degrees)"], np.float32)
    shx = np.asarray(calib["X-shift (pixels)"], np.float32)
    shy = np.asarray(calib["Y-shift (pixels)"], np.float32)
    cpu = (cpu_3d_sample(planes, M, fwhm, S, th, shx, shy, 2)
           if not args.no_cpu_baseline and world == 1 else None)
    # FP32 convention of the RGC launches: 22 ops per evaluated tap, taps per voxel averaged over
    # the sub-pixel phases, RGC launch time from the engine's CUDA events over the timed steps
    taps = taps3d_per_voxel(M, fwhm)
    rgc_s = rgc_timed[0] / 1e3 / args.steps
    ops = n * P * M * h * M * w * M * taps * OPS_PER_TAP
    roofline_fp32 = ({"achieved": ops / rgc_s / 1e12, "peak": FP32_PEAK_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                      "frac": ops / rgc_s / 1e12 / FP32_PEAK_NOMINAL_TFLOPS, "ops_per_step": ops,
                      "taps_per_voxel": taps, "rgc_ms_per_step": rgc_s * 1e3,
                      "convention": "22 FP32 ops per evaluated tap; nominal peak at 1965 MHz"}
                     if rgc_s > 0 else None)
    print(json.dumps({
        "metric": "input Mpx*frames/s (eSRRF 3-D MFM path)", "value": world * mpxf / t_step,
        "unit": "Mpx*frames/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"mfm3d: {P} planes of {w}x{h} x {n} timepoints, M3, radius 1.5, S1, "
                               "AVG+VAR (+TAC2, INT), MP correction, one block",
                   "kernel": "tabulated taps" if args.kernel == "fused" else "plain per-voxel",
                   "timepoints_per_launch": tpl.value},
        "forms": {"batched_timepoints_per_launch_ms": t_step * 1e3,
                  "plain_1_timepoint_per_launch_ms": plain_ms,
                  "plain_1_timepoint_per_launch_mpx_frames_s": mpxf / (plain_ms / 1e3) if plain_ms else None},
        "e2e": {"value": mpxf / e2e, "unit": "Mpx*frames/s", "h2d_bytes_per_step": int(cam.nbytes),
                "d2h_bytes_per_step": int(h_out.numel() * 4)},
        "gpu_launches": launches[0], "roofline_fp32": roofline_fp32, "clocks": clk.summary(),
        "cpu_baseline": cpu}))


def drift_cpu_sample(stack, n):
    """The float64 numpy-FFT restatement (oracle/drift_oracle.py) on n frames, timed."""
    from oracle import drift_oracle as D

    t0 = time.perf_counter()
    D.estimate_drift(stack[:n].astype(np.float64))
    dt = time.perf_counter() - t0
    return {"value": n / dt, "unit": "frames/s", "cores": 1, "kind": "port",
            "sample": f"{n} frames of {stack.shape[2]}x{stack.shape[1]} against the first: numpy FFT "
                      f"(one thread), window, arg-max, quadratic fit; {dt:.2f} s"}


def run_drift(args, world, rank, local):
    """Drift estimation over the headline stack (512x512x500 uint16): one esrrf_estimate_drift call
    per block of 100 frames against the block's first frame, as the live plugin does per SR frame
    (LiveSRRF_optimised_.java:283-288).  Lags |s| <= 31."""
    import ctypes

    import torch

    import esrrf
    from esrrf import synth

    torch.cuda.set_device(local)
    stack = synth.make_stack("fht512", frames=args.frames)
    n, h, w = stack.shape
    blk = args.block or 100
    blocks = [(i, min(blk, n - i)) for i in range(0, n, blk)]
    d = torch.from_numpy(stack.view(np.int16)).to(f"cuda:{local}")
    L = esrrf.lib()
    R = esrrf.drift_window(w, h)
    sx = np.empty(blk, np.float32)
    sy = np.empty(blk, np.float32)
    fp = ctypes.POINTER(ctypes.c_float)
    stream = torch.cuda.current_stream(local)

    def call(ptr, i0, cnt):
        esrrf._lib.check(None, L.esrrf_estimate_drift(
            ctypes.c_void_p(ptr + 2 * i0 * h * w), 1, cnt, w, h, 0, R, sx.ctypes.data_as(fp),
            sy.ctypes.data_as(fp), None, ctypes.c_void_p(stream.cuda_stream)), drift=True)

    def step():
        for i0, cnt in blocks:
            call(d.data_ptr(), i0, cnt)

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    t_step = max_over_ranks(world, e0.elapsed_time(e1) / 1e3 / args.steps)
    # end to end: each block copied from pinned host memory, then estimated
    h_st = torch.from_numpy(stack.view(np.int16)).pin_memory()
    d_blk = torch.empty((blk, h, w), dtype=torch.int16, device=f"cuda:{local}")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i0, cnt in blocks:
        d_blk[:cnt].copy_(h_st[i0:i0 + cnt], non_blocking=True)
        call(d_blk.data_ptr(), 0, cnt)
    e2e = time.perf_counter() - t0
    if rank != 0:
        return
    cpu = None if args.no_cpu_baseline or world > 1 else drift_cpu_sample(stack, 40)
    side = 2 * R + 1
    flop = 2.0 * h * w * side * side * n  # one FMA per pixel per lag
    achieved = flop / t_step / 1e12
    print(json.dumps({
        "metric": "frames/s (drift estimation)", "value": world * n / t_step, "unit": "frames/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"drift512: {w}x{h}x{n} uint16, blocks of {blk}, lags |s| <= {R}, "
                               "reference = each block's first frame",
                   "l2": "frames (262 MB) larger than L2"},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": FP32_PEAK_NOMINAL_TFLOPS,
                     "unit": "TFLOP/s", "frac": achieved / FP32_PEAK_NOMINAL_TFLOPS, "traffic": None,
                     "note": "2 flops per pixel per lag over whole calls (4 kernels + 8 B/frame read "
                             "back); peak = nominal FP32 FMA rate at 1965 MHz"},
        "cpu_baseline": cpu,
        "e2e": {"value": n / e2e, "unit": "frames/s", "h2d_bytes_per_step": int(stack.nbytes),
                "d2h_bytes_per_step": 8 * n},
        "gpu_launches": 4 * len(blocks), "clocks": clk.summary()}))


def run_adjoint(args, world, rank, local):
    """Differentiable eSRRF on 256x256x100, M4: forward (loss) time, loss-and-gradient time, their
    ratio, and a gradient search on (radius, sensitivity, re-blur sigma) beside a grid search."""
    import torch

    import esrrf
    from esrrf import synth

    torch.cuda.set_device(local)
    stack = synth.make_stack("adjoint256").astype(np.float32)
    n, h, w = stack.shape
    M = 4
    adj = esrrf.Adjoint(w, h, n, M, device=local)
    d = torch.from_numpy(stack).to(f"cuda:{local}")
    x0 = (1.5, 2.0, 1.5)
    for _ in range(args.warmup):
        adj.loss(d, *x0)
        adj.loss_and_grad(d, *x0)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            adj.loss(d, *x0)
        torch.cuda.synchronize()
        t_f = (time.perf_counter() - t0) / args.steps
        t0 = time.perf_counter()
        for _ in range(args.steps):
            L, g, gf = adj.loss_and_grad(d, *x0)
        torch.cuda.synchronize()
        t_fb = (time.perf_counter() - t0) / args.steps
    t_f = max_over_ranks(world, t_f)
    t_fb = max_over_ranks(world, t_fb)
    # grid search (forward only) and gradient search
    grid = []
    t0 = time.perf_counter()
    for r in SWEEP_RADII:
        for S in SWEEP_SENS:
            for sg in (1.0, 1.5, 2.0, 3.0):
                grid.append((adj.loss(d, r, S, sg), r, S, sg))
    t_grid = time.perf_counter() - t0
    best = min(grid)
    t0 = time.perf_counter()
    # same domain as the grid: radius 0.5..3.0, S 1..4, sigma 0.5..8
    traj = esrrf.gradient_search(adj, d, 1.0, 2.0, 1.5, steps=25,
                                 bounds=((0.5, 3.0), (1.0, 4.0), (0.5, 8.0)))
    t_gs = time.perf_counter() - t0
    adj.release()
    if rank != 0:
        return
    xg, Lg = traj[-1]
    print(json.dumps({
        "metric": "adjoint time / forward time (loss + all gradients vs loss)", "value": (t_fb - t_f) / t_f,
        "unit": "ratio", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t_fb * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "adjoint256: 256x256x100, M4, AVG, loss = re-blur MSE vs frame mean "
                               "(alpha, beta refit), gradients w.r.t. radius, S, sigma and all 6.6 M input pixels"},
        "forward_ms": t_f * 1e3, "loss_and_grad_ms": t_fb * 1e3,
        "forward_input_mpx_frames_s": n * h * w / 1e6 / t_f,
        "grid_search": {"evaluations": len(grid), "seconds": t_grid, "best_loss": best[0],
                        "best": {"radius": best[1], "S": best[2], "sigma": best[3]}},
        "gradient_search": {"iterations": len(traj) - 1, "seconds": t_gs, "loss": Lg,
                            "x": {"radius": float(xg[0]), "S": float(xg[1]), "sigma": float(xg[2])}},
        "e2e": {"value": (t_fb - t_f) / t_f, "unit": "ratio", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "clocks": clk.summary()}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="fht512", choices=sorted(WORKLOADS))
    ap.add_argument("--kernel", default="fused", choices=["fused", "plain"])
    ap.add_argument("--frames-per-launch", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="quick run: no CPU reference sample and no secondary metrics (profiling runs)")
    ap.add_argument("--frames", type=int, default=None,
                    help="shorter stack (profiling runs); default: the workload's length")
    ap.add_argument("--block", type=int, default=0, help="frames per block override")
    ap.add_argument("--drift", action="store_true",
                    help="fht512/bic512: a seeded per-frame shift in every block (vibration correction)")
    args = ap.parse_args()
    if args.impl == "reference":
        # rank 0 alone times the CPU reference; it takes no collective, so no process group
        run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")))
        return
    world, rank, local = dist_setup()
    try:
        if args.workload == "sweep256":
            run_sweep(args, world, rank, local)
        elif args.workload == "mfm3d":
            run_3d(args, world, rank, local)
        elif args.workload == "adjoint256":
            run_adjoint(args, world, rank, local)
        elif args.workload == "drift512":
            run_drift(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
