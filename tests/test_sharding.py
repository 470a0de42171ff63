"""Sub-database sharding of one answer (kspir_b200/sharding.py) across two
ranks over torch.distributed (gloo, CPU).  The per-rank compute here is the
oracle (test-only backend); the orchestration under test -- shard ranges,
local shares in rank order, one gather to rank 0, packing there -- is the
product's.  The sharded response must equal the unsharded oracle answer."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from kspir_b200 import sharding  # noqa: E402
from oracle import pyoracle as po  # noqa: E402

N = po.N
R, N1, SEED = 4, 128, 401


class OracleShard:
    """Test backend: a rank's share computed by the CPU oracle."""

    def __init__(self, db, c, world, rank):
        lo, hi = sharding.shard_range(R, world, rank)
        words = N * N // 2
        self.db, self.c, self.local = db[lo * words:hi * words], c, hi - lo

    def local_ext(self, query):
        first, _ = po.matrix_vector_mul(self.db, self.local, N1, dict(self.c, query=query))
        out = []
        for j in range(self.local):
            e, _ = po.external_product(first[j * 2 * N:(j + 1) * 2 * N], self.c["rgsw"], ext=np.zeros(2 * N, np.uint64))
            out.append(e)
        return np.stack(out)

    def pack(self, ext_all):
        return po.packing(np.ascontiguousarray(ext_all).reshape(-1), R, self.c["packing"])


def _worker(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        db = po.gen_db(SEED, R, N1)
        c = po.gen_client(SEED, R, N1)
        sa = sharding.ShardedAnswer(OracleShard(db, c, world, rank), R, world, rank, sharding.gather_torch())
        resp = sa.answer(c["query"])
        if rank == 0:
            np.save(os.path.join(outdir, "resp.npy"), resp)
        else:
            assert resp is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_ranges():
    assert sharding.shard_range(16, 4, 2) == (8, 12)
    assert sharding.shard_range(4, 1, 0) == (0, 4)
    for bad in ((16, 3, 0), (4, 8, 0), (16, 0, 0)):
        with pytest.raises(ValueError):
            sharding.shard_range(*bad)


def test_two_rank_gloo_answer_equals_unsharded(tmp_path):
    import torch.multiprocessing as mp
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    got = np.load(tmp_path / "resp.npy")
    db = po.gen_db(SEED, R, N1)
    c = po.gen_client(SEED, R, N1)
    assert np.array_equal(got, po.answer(db, R, N1, c))
