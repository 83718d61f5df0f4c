"""The forward NTT's FP64 butterflies (shmoai_b200/csrc/ntt.cuh: ct_bf_dbl, dbl_centre) restated in C
with IEEE double operations and checked against exact integer arithmetic over all 16 stages at
N = 2^16, at primes at the edges of both FP64 families (just below 2^52/36 without centring; near
2^51, 2^50 and just above 2^52/36 with centring), with a count of quotients outside the exact range
of the 1.5 2^52 rounding and of values at or above 2^53."""
import os
import shutil
import subprocess
import tempfile

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_fp64_forward_butterflies_exact():
    with tempfile.TemporaryDirectory() as d:
        exe = os.path.join(d, "fp64_ntt_check")
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe, os.path.join(HERE, "native", "fp64_ntt_check.c"),
                        "-lm"], check=True)
        r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout
    lines = [l for l in r.stdout.splitlines() if l.startswith("q=")]
    assert len(lines) == 6
    for l in lines:
        assert "mismatches 0, range violations 0" in l, l
