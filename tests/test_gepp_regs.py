"""The Newton fast path's register GEPP (row swaps written as bitwise blends,
so that a 5 x 5 block stays in registers) gives the full-matrix GEPP's
solution bit for bit, row swaps and small pivots included.  Both come from
the library's own header, compiled for the host."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "zoomy-dmplex_b200", "csrc")


def test_register_gepp_matches_full_gepp(tmp_path):
    exe = str(tmp_path / "gepp_regs_check")
    cc = subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC,
                         os.path.join(ROOT, "tests", "gepp_regs_check.cpp"), "-o", exe],
                        capture_output=True, text=True)
    if cc.returncode != 0:
        pytest.fail(cc.stderr)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    words = r.stdout.split()
    swaps, singular = int(words[1]), int(words[3])
    assert swaps > 10000 and singular > 1000, r.stdout
