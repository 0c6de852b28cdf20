"""CPU tests of how bench.py ties its quoted ncu figures to the kernel sources they were taken of.

The bench quotes a kernel's DRAM traffic and warp instructions per frame from its committed
profile summary only while the kernel sources' code hashes to the summary's `source_sha:` line
(comments and blank lines do not count, code does).
"""
import importlib.util
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    argv = sys.argv
    sys.argv = ["bench.py"]
    try:
        spec.loader.exec_module(mod)
    finally:
        sys.argv = argv
    return mod


def test_code_hash_ignores_comments_not_code(bench):
    src = "int f(int x) {\n    return x + 1;  // one more\n}\n"
    commented = "/* header\n   lines */\nint f(int x) {\n\n    return x + 1;   // a different note\n}\n"
    changed = "int f(int x) {\n    return x + 2;  // one more\n}\n"
    assert bench._code_only(src) == bench._code_only(commented)
    assert bench._code_only(src) != bench._code_only(changed)


@pytest.mark.parametrize("kernel", sorted(["rgc_fused_fht512", "rgc_fused_bic512", "rgc_fused_fht512_drift"]))
def test_committed_summaries_match_the_current_kernel_code(bench, kernel):
    """Every summary the bench quotes was captured from the kernel code in the tree, and carries
    both figures the bench reads."""
    assert bench.summary_stale(kernel) is None, bench.summary_stale(kernel)
    assert bench.read_traffic_summary(kernel) > 0
    assert bench.read_traffic_summary(kernel, "warp_instructions_per_frame") > 0


def test_a_changed_kernel_makes_its_summary_stale(bench, monkeypatch):
    real = bench.source_sha
    monkeypatch.setattr(bench, "source_sha", lambda k: "0" * 16 if k == "rgc_fused_fht512" else real(k))
    msg = bench.summary_stale("rgc_fused_fht512")
    assert msg and "re-capture" in msg
    assert bench.summary_stale("rgc_fused_bic512") is None


@pytest.mark.parametrize("world", [1, 2, 4, 8])
def test_ranks_take_disjoint_contiguous_runs_of_blocks(bench, esrrf_mod, world):
    """Under torchrun each rank reconstructs its run of blocks of a world-size times longer stack
    (weak scaling); the runs come from the library's planner, cover every block once, are
    contiguous, and all have the length of the one-GPU workload (5 blocks of 100 frames)."""
    runs = [bench.shard_blocks(world, r, 5, 100) for r in range(world)]
    assert sorted(b for run in runs for b in run) == list(range(5 * world))
    for run in runs:
        assert len(run) == 5 and run == list(range(run[0], run[0] + 5))
