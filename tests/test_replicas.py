"""The multi-GPU path of bench.py (replicas, no collective in the data path)
with world size 2 on CPU over gloo: per-rank rays and the max/sum reduction
of the ranks' times and bounce counts."""
import os
import socket
import sys

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        t, b = bench._max_over_ranks(1.5 + rank, 100 * (rank + 1), torch.device("cpu"), world)
        from billardballraytracing3d_b200 import scenes
        _, o, d, *_ = scenes.workload("tetra_spheres", 2048)
        ro, rd = bench.replica_rays("tetra_spheres", o, d, rank)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), t=t, b=b, o=ro, d=rd)
    finally:
        dist.destroy_process_group()


def test_replicas_world_size_2_gloo(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    r0, r1 = (np.load(tmp_path / f"r{k}.npz") for k in range(world))
    # time = max over ranks, work = sum over ranks, the same on every rank
    for r in (r0, r1):
        assert float(r["t"]) == 2.5 and int(r["b"]) == 300
    # rank 0 traces the workload's own rays, rank 1 its own seeded set of the same source
    from billardballraytracing3d_b200 import scenes
    _, o, d, *_ = scenes.workload("tetra_spheres", 2048)
    assert np.array_equal(r0["o"], o) and np.array_equal(r0["d"], d)
    assert r1["o"].shape == o.shape and not np.array_equal(r1["o"], o)
    assert np.allclose(np.linalg.norm(r1["d"], axis=1), 1.0)
