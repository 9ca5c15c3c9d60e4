"""Host logic of bench.py's multi-process (replica) mode, on CPU with two
gloo ranks: process-group set-up from the torchrun environment, the barrier
and max-over-ranks timing reduction, and the reference arm's rank handling."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE=str(world), RANK=str(rank),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    import torch.distributed as dist
    w, r, local = bench.dist_setup(backend="gloo")
    assert (w, r, local) == (world, rank, rank)
    got = bench.barrier_max(w, 1.5 + rank)          # per-rank timings 1.5, 2.5, ...
    # the reference arm does no work on ranks other than 0
    if r:
        assert bench.run_reference(None, w, r) is None
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, f"r{rank}.txt"), "w") as f:
        f.write(repr(got))


def test_replica_max_over_ranks(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    port = _free_port()
    mp.start_processes(_rank_main, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    vals = [float(open(tmp_path / f"r{r}.txt").read()) for r in range(world)]
    assert vals == [2.5, 2.5]


def test_single_process_needs_no_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK"):
        monkeypatch.delenv(k, raising=False)
    assert bench.dist_setup() == (1, 0, 0)
    assert bench.barrier_max(1, 3.25) == 3.25
