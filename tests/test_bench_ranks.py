"""bench.py's multi-rank logic on CPU with the gloo backend (world size 2): the max-over-ranks timing that
turns per-replica device times into the job's time, and the reference arm running on rank 0 only."""
import json
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * rank], world, torch.device("cpu"))
        ref_line = bench.run_reference(None, rank, world) if rank != 0 else "rank0"
        (Path(out_dir) / f"r{rank}.json").write_text(json.dumps({"max": got, "ref": ref_line}))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_rank0_only_reference(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for rank in range(2):
        d = json.loads((tmp_path / f"r{rank}.json").read_text())
        assert d["max"] == [2.0, 10.0, 0.5]
    assert json.loads((tmp_path / "r1.json").read_text())["ref"] is None


def test_single_rank_max_is_identity():
    sys.path.insert(0, str(ROOT))
    import bench
    assert bench.max_over_ranks([3.0, 4.0], 1, None) == [3.0, 4.0]
