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
