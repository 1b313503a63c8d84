"""Multi-rank host logic on CPU: two gloo ranks render their shards of a frame with the oracle
(distinct Philox subsequences) and combine the accumulation buffers with an all-reduce, exactly
as bench.py does with NCCL on GPUs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import multigpu


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    for sub in ("gpu-path-tracer_b200", "oracle"):
        sys.path.insert(0, os.path.join(os.path.dirname(here), sub))
    import oracle
    import scenes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.cornell_box(1)
        o = oracle.OracleScene(s)
        cam = scenes.scene_camera(s, 16, 16)
        spf = 4 * 16 * 16
        res = o.render(cam, 16, 16, 4, 6, True, threads=2, rng_offset=multigpu.rank_rng_offset(rank, spf))
        acc = torch.from_numpy(res["accumulation"].copy())
        local = acc.clone()
        multigpu.combine_accumulation(acc, dist)
        times = multigpu.max_over_ranks([float(rank + 1), 10.0 - rank], dist)
        if rank == 0:
            np.save(out + "_combined.npy", acc.numpy())
            np.save(out + "_times.npy", np.array(times))
        np.save(out + f"_local{rank}.npy", local.numpy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_combine(tmp_path):
    out = str(tmp_path / "mr")
    mp.start_processes(_worker, args=(2, free_port(), out), nprocs=2, start_method="spawn", join=True)
    combined = np.load(out + "_combined.npy")
    l0, l1 = np.load(out + "_local0.npy"), np.load(out + "_local1.npy")
    assert np.array_equal(combined, l0 + l1)
    assert not np.array_equal(l0, l1)  # disjoint Philox subsequences
    assert np.load(out + "_times.npy").tolist() == [2.0, 10.0]


def test_rank_offsets_are_disjoint():
    spf = 1920 * 1080 * 64
    offs = [multigpu.rank_rng_offset(r, spf) for r in range(8)]
    assert offs == [r * spf for r in range(8)]
    assert multigpu.combined_samples_per_pixel(64, 8) == 512
    with pytest.raises(ValueError):
        multigpu.rank_rng_offset(-1, spf)
