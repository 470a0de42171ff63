"""Device-side failure detection: the bounded waits of the database scan.

Every mbarrier wait of the scan kernels gives up after a time limit, records
an error word and returns, so a lost copy ends in KSPIR_ERR_TIMEOUT instead of
a hung GPU.  kspir_debug_scan_fault makes that happen on purpose without any
fault: the next single-answer scan does not request the bytes of one work
item, and the wait for them runs out (limit shortened to 1 ms here).  The
context must then answer correctly again.
"""
import time

import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu


def test_scan_wait_runs_out_and_context_recovers():
    r, N1 = 2, 128
    db = po.gen_db(301, r, N1)
    c = po.gen_client(302, r, N1)
    want = po.answer(db, r, N1, c)
    with kb.Context(r, N1) as ctx:
        ctx.upload_db(db)
        ctx.upload_perms(c["perms"])
        ctx.upload_client(0, c["baby"], c["giant"], c["packing"], c["rgsw"])
        assert np.array_equal(ctx.answer(0, c["query"]), want)
        ctx.debug_scan_fault(wait_limit_ns=1_000_000, skip_item=3)
        t0 = time.perf_counter()
        with pytest.raises(kb.KspirError) as ei:
            ctx.answer(0, c["query"])
        assert ei.value.code == kb.native.ERR_TIMEOUT
        assert time.perf_counter() - t0 < 10
        # the injected failure applied to one launch; the next answers are exact
        assert np.array_equal(ctx.answer(0, c["query"]), want)
        ctx.debug_scan_fault()   # default limit again
        assert np.array_equal(ctx.answer(0, c["query"]), want)


def test_scan_fault_rejects_bad_item():
    with kb.Context(1, 128) as ctx:
        with pytest.raises(kb.KspirError):
            ctx.debug_scan_fault(skip_item=-2)
