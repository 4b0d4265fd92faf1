"""Training-set generation as replicas (learned.generate_distributed): two
gloo ranks on CPU, each running its strided share of the seeds through a
stand-in sample function (the SCF itself needs a GPU), one host barrier, and
rank 0 merging the records.  Checks that every seed is generated exactly
once, that the skipped seed is recorded, that a rerun resumes without
regenerating, and that load_samples returns the set in seed order."""
import json
import os
import socket
from pathlib import Path

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

from parsec_python_b200 import learned  # noqa: E402

SEEDS = list(range(3, 14))
BAD = 8


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def fake_sample(seed: int, family: str):
    if seed == BAD:
        raise ValueError("Bounds are incorrect")
    n = 4 * 5 * 6
    dom = {"nx": 4, "ny": 5, "nz": 6, "h": 0.4, "radius": 1.0}
    rs = np.full(n, seed, np.float32)
    return rs, rs + 0.5, rs - 0.25, dom, 10 + seed


def _worker(rank: int, world: int, port: int, out_dir: str, calls_dir: str) -> None:
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})

    def counted(seed, family):
        Path(calls_dir, f"{rank}_{seed}").write_text("")
        return fake_sample(seed, family)

    learned.generate_distributed("water", SEEDS, Path(out_dir), sample_fn=counted, timeout_s=120)


def _run(world, out, calls):
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, str(out), str(calls)), nprocs=world, join=True,
                       start_method="spawn")


def test_partition_covers_every_seed_once():
    for world in (1, 2, 3, 8):
        parts = [learned.partition_seeds(SEEDS, r, world) for r in range(world)]
        flat = [s for p in parts for s in p]
        assert sorted(flat) == SEEDS and len(flat) == len(set(flat))
        assert max(map(len, parts)) - min(map(len, parts)) <= 1
    with pytest.raises(ValueError):
        learned.partition_seeds(SEEDS, 2, 2)


def test_two_gloo_replicas_generate_the_set(tmp_path):
    out, calls = tmp_path / "set", tmp_path / "calls"
    calls.mkdir()
    _run(2, out, calls)
    man = json.loads((out / "manifest.json").read_text())
    assert man["seeds"] == [s for s in SEEDS if s != BAD] and man["skipped"] == [BAD] and man["world"] == 2
    made = sorted(p.name for p in calls.iterdir())
    # each seed ran once, on the rank the strided partition gives it
    assert made == sorted(f"{SEEDS.index(s) % 2}_{s}" for s in SEEDS)
    for r in range(2):
        rec = json.loads((out / f"manifest_rank{r}.json").read_text())
        assert sorted(rec["done"] + rec["skipped"]) == learned.partition_seeds(SEEDS, r, 2)
    dom, samples, seeds = learned.load_samples(out, 3)
    assert seeds == [3, 4, 5] and dom["nx"] == 4
    for sd, (rs, vl, dt) in zip(seeds, samples):
        assert rs.dtype == torch.float64 and dt.dtype == torch.float32
        assert float(rs[0]) == sd and float(vl[-1]) == sd + 0.5 and float(dt[7]) == sd - 0.25
    # a rerun keeps the files and only retries the skipped seed
    for p in calls.iterdir():
        p.unlink()
    _run(2, out, calls)
    assert sorted(p.name for p in calls.iterdir()) == [f"{SEEDS.index(BAD) % 2}_{BAD}"]


def test_merge_rejects_duplicate_and_missing_records(tmp_path):
    for r, done in ((0, [1, 2]), (1, [2, 3])):
        (tmp_path / f"manifest_rank{r}.json").write_text(
            json.dumps({"rank": r, "world": 2, "family": "water", "done": done, "skipped": [], "seconds": 0.0}))
    with pytest.raises(ValueError):
        learned.merge_manifests(tmp_path, 2)
    with pytest.raises(FileNotFoundError):
        learned.merge_manifests(tmp_path, 3)
