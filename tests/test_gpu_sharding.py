"""The GPU shares of a sharded answer (kspir_b200/sharding.GpuShard): two ranks'
shares computed on this GPU, gathered in rank order and packed on rank 0, give
the unsharded response word for word.  (The collective itself is covered by
tests/test_sharding.py over gloo; every run here has one GPU.)"""
import numpy as np
import pytest

import kspir_b200 as kb
from kspir_b200 import sharding
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
R, N1 = 8, 128


def test_gpu_shards_compose_to_the_full_answer():
    db = po.gen_db(411, R, N1)
    c = po.gen_client(411, R, N1)
    shards = [sharding.GpuShard(db, R, N1, 2, g, c["perms"], c) for g in range(2)]
    try:
        parts = [s.local_ext(c["query"]) for s in shards]
        sa = sharding.ShardedAnswer(shards[0], R, 2, 0, lambda local: parts)
        got = sa.answer(c["query"])
    finally:
        for s in shards:
            s.close()
    with kb.Context(R, N1) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        assert np.array_equal(got, ctx.answer(0, c["query"]))
    assert np.array_equal(got, po.answer(db, R, N1, c))


def _gpu_worker(rank, world, port, outdir):
    # two processes, each with its own context on this GPU: the shares are
    # computed independently (no kernel waits on another process) and gathered
    # to rank 0 over gloo, as the multi-GPU job does over NCCL
    import datetime
    import os

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    shard = None
    try:
        db = po.gen_db(421, R, N1)
        c = po.gen_client(421, R, N1)
        shard = sharding.GpuShard(db, R, N1, world, rank, c["perms"], c)
        resp = sharding.ShardedAnswer(shard, R, world, rank, sharding.gather_torch()).answer(c["query"])
        if rank == 0:
            np.save(os.path.join(outdir, "resp.npy"), resp)
        else:
            assert resp is None
    finally:
        if shard is not None:
            shard.close()
        dist.destroy_process_group()


def test_two_processes_gloo_gather_equals_unsharded(tmp_path):
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.spawn(_gpu_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    got = np.load(tmp_path / "resp.npy")
    db = po.gen_db(421, R, N1)
    c = po.gen_client(421, R, N1)
    assert np.array_equal(got, po.answer(db, R, N1, c))
