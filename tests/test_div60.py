"""The MP5 reconstruction's division-free x / 60 (div60, axb_recon.cuh)
gives the correctly rounded quotient: the same FMA sequence compiled for the
host (gcc, IEEE double, libm fma) against x / 60 on 26 million values."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no gcc")
def test_div60_is_the_correctly_rounded_quotient():
    out = os.path.join(HERE, "_build")
    os.makedirs(out, exist_ok=True)
    exe = os.path.join(out, "div60_check")
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-o", exe,
                    os.path.join(HERE, "div60_check.c"), "-lm"], check=True)
    r = subprocess.run([exe, "20000000"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert " 0 mismatches" in r.stdout
