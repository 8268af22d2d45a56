"""The multi-rank logic of bench.py on CPU: two gloo ranks (torch.distributed
over 127.0.0.1), no GPU.  Covers the per-rank guide sets of the weak-scaling
run and the max-over-ranks reduction of the timed values."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "cas-offinder-rust-old_b200"))

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r pretends its device time was 10 + r ms and its e2e 5 - r s
        got = bench.max_over_ranks(dist, [10.0 + rank, 5.0 - rank], "cpu")
        pats = bench.rank_patterns(["ACGT" * 5 + "NNN"] * 4, rank)
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(repr((got, pats)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = eval((tmp_path / "rank0.txt").read_text())
    r1 = eval((tmp_path / "rank1.txt").read_text())
    # every rank sees the slowest rank's values
    assert r0[0] == r1[0] == [11.0, 5.0]
    # rank 0 keeps the workload's guides; rank 1 brings its own, same shape
    assert r0[1] == ["ACGT" * 5 + "NNN"] * 4
    assert r1[1] != r0[1] and len(r1[1]) == 4
    assert all(len(p) == 23 and p.endswith("NNN") for p in r1[1])


def test_rank_patterns_deterministic():
    a = bench.rank_patterns(["N" * 23] * 3, 2)
    b = bench.rank_patterns(["N" * 23] * 3, 2)
    c = bench.rank_patterns(["N" * 23] * 3, 3)
    assert a == b and a != c


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(None, [1, 2.5], "cpu") == [1.0, 2.5]


def test_reference_arm_runs_on_rank_zero_only():
    class A:  # the arguments run_reference reads before its rank check
        pass
    assert bench.run_reference(A(), 1, 2) is None
