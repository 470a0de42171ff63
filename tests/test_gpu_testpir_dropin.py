"""The drop-in: the reference's unmodified tests/test-pir.cpp, linked with
kspir_b200/cpp/reference_api.cpp in place of the reference's three answer
functions and its two preprocessing functions (database_tobsgsntt,
database_tocrt; built by `make -C oracle testpir-gpu`), preprocesses its
database and runs its online answer on the GPU, and recovers the planted
record like the reference build does."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "oracle", "_ref", "test-pir-gpu")

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(BIN), reason="oracle/_ref/test-pir-gpu not built (needs the reference tree)")
def test_unmodified_testpir_recovers_the_record_through_the_gpu():
    out = subprocess.run([BIN], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    want = "the recovered result = [" + ", ".join(str(i) for i in range(1, 17)) + ", ..., 4096]"
    assert want in out.stdout, out.stdout[-2000:]
    assert "online server response costs" in out.stdout
    assert "server preprocessing costs" in out.stdout


INPLACE = os.path.join(ROOT, "oracle", "_ref", "dropin-inplace")


@pytest.mark.skipif(not os.path.exists(INPLACE), reason="oracle/_ref/dropin-inplace not built (needs the reference tree)")
def test_dropin_follows_objects_rewritten_in_place():
    # tests/dropin_inplace.cpp: the RGSW query re-keyed in place and the
    # database rebuilt in place (same addresses) must change the answer, and
    # packingRLWEs leaves rlwes[0] equal to the response, as the reference does
    out = subprocess.run([INPLACE], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    assert "dropin-inplace: ok" in out.stdout
