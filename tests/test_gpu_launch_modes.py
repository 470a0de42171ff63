"""The answer is the same in every launch mode: CUDA graphs on or off
(KSPIR_NO_GRAPHS), programmatic dependent launch on or off (KSPIR_NO_PDL),
and single answers as separate kernels or as the one fused kernel
(KSPIR_FUSED).  The modes only change how the same arithmetic is launched,
and each context reads them when it is created."""
import os

import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("env", [{}, {"KSPIR_NO_GRAPHS": "1"}, {"KSPIR_NO_PDL": "1"},
                                 {"KSPIR_NO_GRAPHS": "1", "KSPIR_NO_PDL": "1"}, {"KSPIR_FUSED": "1"}],
                         ids=["default", "no-graphs", "no-pdl", "neither", "fused"])
def test_launch_modes_answer_alike(env, monkeypatch):
    for k, v in env.items():
        monkeypatch.setenv(k, v)
    r, N1 = 4, 128
    db = po.gen_db(401, r, N1)
    c = po.gen_client(402, r, N1)
    want = po.answer(db, r, N1, c)
    rng = np.random.default_rng(403)
    q = np.empty((3, 4 * po.N), np.uint64)
    q[:, :2 * po.N] = rng.integers(0, po.CRTMOD, size=(3, 2 * po.N), dtype=np.uint64)
    q[:, 2 * po.N:] = rng.integers(0, po.BSMOD, size=(3, 2 * po.N), dtype=np.uint64)
    with kb.Context(r, N1, max_clients=1, max_inflight=4) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        for _ in range(2):   # graph capture on the first call, replay on the second
            assert np.array_equal(ctx.answer(0, c["query"]), want)
        got = ctx.answer_batch(np.zeros(3, np.int32), q)
        for i in range(3):
            assert np.array_equal(got[i], po.answer(db, r, N1, dict(c, query=q[i]))), f"query {i}"
