"""The multi-process plumbing of bench.py on CPU: two gloo ranks initialise
from the torchrun environment, meet at the barrier, agree on the maximum of
their step times (the bench reports the slowest rank), and only rank 0 runs
the reference arm."""
import os
import socket
import sys
from pathlib import Path

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, str(ROOT))
    import bench
    import torch.distributed as dist

    r, local, w = bench.dist_init()
    assert (r, local, w) == (rank, rank, world)
    assert dist.get_backend() == "gloo"
    bench.barrier(w)
    worst = bench.allmax(1.0 + rank, w)

    class Args:
        steps, warmup, gpus = 1, 0, world

    # every rank but 0 leaves the reference arm at once, without work
    if rank != 0:
        bench.run_reference_arm(Args, rank, w)
    bench.barrier(w)
    Path(out_dir, f"rank{rank}.txt").write_text(repr(worst))
    dist.destroy_process_group()


def test_two_gloo_ranks_share_barrier_and_max(tmp_path):
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    for rank in range(2):
        assert float((tmp_path / f"rank{rank}.txt").read_text()) == 2.0
