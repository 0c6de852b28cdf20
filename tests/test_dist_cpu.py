"""The multi-GPU bench path on CPU: world_size-2 gloo ranks exercise the barrier and the
max-over-ranks timing reduction that bench.py uses under torchrun (rolling blocks are
independent, so there is no data-path collective to test)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dist.barrier()
        t = torch.tensor([1.0 + rank], dtype=torch.float64)  # per-rank step time
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        out[rank] = float(t.item())
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_max_timing():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        assert dict(out) == {0: 2.0, 1: 2.0}


def test_bench_value_is_whole_job_throughput():
    """value = all ranks' input pixel-frames / max step time (weak scaling)."""
    import importlib.util
    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(os.path.dirname(__file__)), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.taps_per_pixel(4, 1.5) == 254
    assert bench.taps_per_pixel(5, 1.5) == 394
    assert bench.max_over_ranks(1, 3.5) == 3.5


def test_bench_bicubic_tap_count():
    """The bicubic path's taps per output pixel (its FP32 roofline convention): 64 at M4, radius
    1.5, and the same count at another interior cell by a direct walk of the reference's loop
    (liveSRRF.cl:238-401 geometry, FP32)."""
    import importlib.util
    import numpy as np
    spec = importlib.util.spec_from_file_location(
        "bench", os.path.join(os.path.dirname(os.path.dirname(__file__)), "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert bench.bic_taps_per_pixel(4, 1.5) == 64.0
    f = np.float32
    for M, fwhm in ((4, 1.5), (3, 2.5), (2, 1.0)):
        sigma = f(fwhm) / f(2.354)
        radius = f(int(f(4) * sigma)) / f(2) + f(1)
        tSO = f(2) * sigma + f(1)
        r0, r1 = -int(f(2) * radius), int(f(2) * radius + f(1))
        total = 0
        cell = 200
        for yM in range(cell * M, cell * M + M):
            for xM in range(cell * M, cell * M + M):
                xc, yc = f((xM + 0.5) / M), f((yM + 0.5) / M)
                kx, ky = int(f(2) * xc), int(f(2) * yc)
                for j in range(r0, r1 + 1):
                    for i in range(r0, r1 + 1):
                        dx = f(f(kx + i) / f(2)) - xc
                        dy = f(f(ky + j) / f(2)) - yc
                        d = np.sqrt(f(dx * dx + dy * dy))
                        total += d != 0 and d <= tSO
        assert abs(total / (M * M) - bench.bic_taps_per_pixel(M, fwhm)) < 1e-9, (M, fwhm)
