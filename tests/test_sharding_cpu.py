"""Host logic of the multi-GPU split (z-slabs of one grid, LPT over a batch of meshes) and its
gather, run as two gloo ranks on the CPU with the oracle computing each rank's slab."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from stl2sdf import sharding


def test_zslab_bounds_cover_every_layer_once():
    for nz in (1, 2, 7, 64, 129):
        for world in (1, 2, 3, 4, 8):
            got = [sharding.zslab_bounds(nz, world, r) for r in range(world)]
            layers = [k for b in got if b is not None for k in range(b[0], b[1] + 1)]
            assert layers == list(range(nz))
            sizes = [b[1] - b[0] + 1 for b in got if b is not None]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        sharding.zslab_bounds(10, 2, 2)


def test_lpt_assign_is_balanced_and_deterministic():
    rng = np.random.default_rng(3)
    works = [sharding.mesh_work(int(k) ** 3, int(n)) for k, n in zip(rng.integers(32, 161, 256),
                                                                     rng.integers(320, 400_000, 256))]
    for world in (1, 2, 4, 8):
        plan = sharding.lpt_assign(works, world)
        assert plan == sharding.lpt_assign(works, world)
        assert sorted(i for p in plan for i in p) == list(range(len(works)))
        loads = [sum(works[i] for i in p) for p in plan]
        assert max(loads) - min(loads) <= max(works)  # LPT bound: within the largest item


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    import conftest  # noqa: F401  (import paths)
    import torch.distributed as dist

    import oracle
    from stl2sdf import DataImport
    from workloads import synthetic

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        X, IEN = DataImport.roundtrip_float32(*synthetic.icosphere(2, jitter=0.01, seed=0))
        g = oracle.grid(X.min(0), X.max(0), 17 - 7, 3)
        o, N, h = g["origin"], g["N"], g["h"]
        layer = int((N[0] + 1) * (N[1] + 1))

        def compute(k0, k1):
            nodes = np.arange(k0 * layer, (k1 + 1) * layer, dtype=np.int64)
            d, _, _ = oracle.distances(X, IEN, o, h, N, nodes=nodes, nthreads=1)
            s = oracle.signs(X, IEN, o, h, N, nodes=nodes, nthreads=1)["sign"]
            return d * s

        full = sharding.sdf_zslab(X, IEN, o, h, N, compute=compute)
        if rank == 0:
            d, _, _ = oracle.distances(X, IEN, o, h, N, nthreads=1)
            s = oracle.signs(X, IEN, o, h, N, nthreads=1)["sign"]
            np.save(out_path, np.stack([full, d * s]))
        else:
            assert full is None
    finally:
        dist.destroy_process_group()


def test_zslab_gather_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    out = str(tmp_path / "full.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    got, want = np.load(out)
    assert np.array_equal(got, want)


def test_local_device_follows_the_launcher(monkeypatch):
    """Without an explicit device every rank builds its context on its own GPU (LOCAL_RANK)."""
    monkeypatch.setenv("LOCAL_RANK", "3")
    assert sharding.local_device() == 3
    monkeypatch.delenv("LOCAL_RANK")
    assert sharding.local_device() == 0
    assert sharding.local_device(5) == 5
    assert sharding.local_device("cuda:2") == 2

    class Dev:
        index = 6

    assert sharding.local_device(Dev()) == 6
