"""Host-planner helpers checked against their direct definitions: a C++
test (tests/host/plan_helpers_test.cpp) built with g++ against the product's
plan.cpp and run here.  No GPU."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "ifgf_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_plan_helpers_match_their_definitions(tmp_path):
    exe = str(tmp_path / "plan_helpers_test")
    subprocess.run(["g++", "-O2", "-std=c++17", "-pthread", "-I", CSRC,
                    os.path.join(ROOT, "tests", "host", "plan_helpers_test.cpp"),
                    os.path.join(CSRC, "plan.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert r.stdout.strip().endswith("OK")
