"""GPU: the C++ drop-in (include/dft_b200.hpp) inside a program built from the reference's
own sources: each reference call is compared with its dftb200:: replacement in-process."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "oracle", "_ref", "shim_demo")


def test_reference_program_with_dropin():
    if not os.path.exists(DEMO):
        pytest.skip("oracle/_ref/shim_demo not built (needs the reference tree at build time)")
    r = subprocess.run([DEMO], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr[-2000:]
    assert "all ok" in r.stdout
