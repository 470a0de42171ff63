"""Offline key derivation on the device (kspir_gen_autokey_from_offline):
the reference's genAutoKeyFromOffline (twosteps.cpp:1749-1864) with its key
switch evalAutoRNSKey (twosteps.cpp:1587-1743) and the key parameters of
tests/test-two-steps-key.cpp:149-155.  Integer work: every output key map
must equal the reference's word for word -- against the committed golden
digests (made by tests/golden/make_golden.py from the reference build) and,
where the reference build is present, against it directly."""
import hashlib
import json
import os

import numpy as np
import pytest

import kspir_b200 as kb
from oracle import pyoracle as po

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("case", GOLDEN["offline"], ids=lambda c: f"N1_{c['N1']}")
def test_offline_derivation_matches_reference(case):
    keys = po.gen_offline_keys(case["seed"])
    assert {k: sha(v) for k, v in keys.items()} == case["inputs_sha"]
    with kb.Context(2, case["N1"]) as ctx:
        got = ctx.gen_autokey_from_offline(keys["offline1"], keys["offline2"], keys["auto1"], keys["auto2"])
    if po.ref_available():
        want = po.ref_gen_autokey_from_offline(case["N1"], keys)
        for k in ("chain1", "chain2", "baby", "giant"):
            assert np.array_equal(got[k], want[k]), f"{k}: {int(np.count_nonzero(got[k] != want[k]))} words differ"
    for k in ("chain1", "chain2", "baby", "giant"):
        assert sha(got[k]) == case[k + "_sha"], k
    N1, N = case["N1"], po.N
    # the reference leaves the bsMod rows of every derived baby key zero
    assert not got["baby"].reshape(N1 - 1, 6, 2, N)[:, 3:].any()
    assert got["device_ms"] > 0


def test_offline_derivation_rejects_bad_words():
    keys = po.gen_offline_keys(43)
    bad = keys["auto2"].copy()
    bad[3 * 2 * po.N + 5] = po.AUXMOD        # a row mod auxMod holding auxMod
    with kb.Context(1, 64) as ctx:
        with pytest.raises(kb.KspirError) as ei:
            ctx.gen_autokey_from_offline(keys["offline1"], keys["offline2"], keys["auto1"], bad)
        assert ei.value.code == kb.native.ERR_INVALID_ARG
