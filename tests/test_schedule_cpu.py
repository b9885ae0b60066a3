"""The general SGM pass schedule (thundervision_b200/csrc/paths.cpp), built
with g++: walks inside the image, disjoint cells within a pass, and the
deferred-row bookkeeping of the reference table's repeated walks, for both
tables, 4 and 8 paths, landscape and portrait sizes."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_pass_schedule_bookkeeping(tmp_path):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path / "schedule_test")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I/usr/local/cuda/include",
                    "-I" + os.path.join(ROOT, "thundervision_b200", "csrc"), "-I" + os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "schedule_test.cpp"),
                    os.path.join(ROOT, "thundervision_b200", "csrc", "paths.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "schedule: ok" in r.stdout
