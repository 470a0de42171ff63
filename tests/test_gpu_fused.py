"""The single answer as one kernel (k_answer.cuh, kspir_set_fused): one
cooperative launch in which a key-switch warp group runs the query side, the
giant steps, the external products and the packing tree from a dependency
queue while the scan warps stream the database.  Integer work: every response
must equal the oracle's (and the separate kernels') word for word, at every
shape of the packing tree (r = 1, 2, 8, 16: no level, one, an odd and an even
number of levels), back to back without host synchronisation, and after an
injected wait that runs out."""
import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
N = po.N


def make_ctx(r, db, c, **kw):
    ctx = kb.Context(r, 128, **kw)
    ctx.upload_db(db)
    ctx.upload_perms(c["perms"])
    ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
    ctx.set_fused(True)
    assert ctx.fused
    return ctx


@pytest.mark.parametrize("r", [1, 2, 8, 16])
def test_fused_answer_matches_oracle(r):
    db = po.gen_db(501 + r, r, 128)
    c = po.gen_client(502 + r, r, 128)
    want, bsgs, ext = po.answer(db, r, 128, c, with_stages=True)
    with make_ctx(r, db, c) as ctx:
        got = ctx.answer(0, c["query"])
        assert np.array_equal(ctx.fetch_stage(kb.STAGE_RESULT), bsgs), "first-dimension results"
        if r <= 2:   # from two packing levels on, the tree reuses the external products' buffer
            assert np.array_equal(ctx.fetch_stage(kb.STAGE_EXT), ext), "external products"
        assert np.array_equal(got, want), "response"
        tot, ph = ctx.last_timing()
        assert tot > 0 and all(p >= 0 for p in ph)
        # the same context with the separate kernels
        ctx.set_fused(False)
        assert np.array_equal(ctx.answer(0, c["query"]), want)


def test_fused_many_queries_and_back_to_back():
    torch = pytest.importorskip("torch")
    r, n = 16, 24
    db = po.gen_db(511, r, 128)
    c = po.gen_client(512, r, 128)
    rng = np.random.default_rng(513)
    q = np.empty((n, 4 * N), np.uint64)
    q[:, :2 * N] = rng.integers(0, po.CRTMOD, size=(n, 2 * N), dtype=np.uint64)
    q[:, 2 * N:] = rng.integers(0, po.BSMOD, size=(n, 2 * N), dtype=np.uint64)
    with make_ctx(r, db, c) as ctx:
        dq = torch.from_numpy(q.view(np.int64).copy()).cuda()
        out = torch.zeros((n, 2 * N), dtype=torch.int64, device="cuda")
        stream = torch.cuda.Stream()
        torch.cuda.synchronize()
        for i in range(n):
            ctx.answer_device(0, dq[i].data_ptr(), out[i].data_ptr(), stream.cuda_stream)
        ctx.sync()
        got = out.cpu().numpy().view(np.uint64)
        ctx.set_fused(False)
        for i in range(n):
            assert np.array_equal(got[i], ctx.answer(0, q[i])), f"query {i}"
    for i in (0, n - 1):
        assert np.array_equal(got[i], po.answer(db, r, 128, dict(c, query=q[i])))


def test_fused_wait_runs_out_and_context_recovers():
    r = 2
    db = po.gen_db(521, r, 128)
    c = po.gen_client(522, r, 128)
    want = po.answer(db, r, 128, c)
    with make_ctx(r, db, c) as ctx:
        assert np.array_equal(ctx.answer(0, c["query"]), want)
        ctx.debug_scan_fault(wait_limit_ns=1_000_000, skip_item=2)
        with pytest.raises(kb.KspirError) as ei:
            ctx.answer(0, c["query"])
        assert ei.value.code == kb.native.ERR_TIMEOUT
        assert np.array_equal(ctx.answer(0, c["query"]), want)
        ctx.debug_scan_fault()
        assert np.array_equal(ctx.answer(0, c["query"]), want)


def test_fused_is_refused_where_unavailable():
    with kb.Context(1, 64) as ctx:
        with pytest.raises(kb.KspirError) as ei:
            ctx.set_fused(True)
        assert ei.value.code == kb.native.ERR_NOT_READY
        assert not ctx.fused
