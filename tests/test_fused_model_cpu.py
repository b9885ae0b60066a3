"""The fused path's arithmetic for the reference semantics, checked on the CPU
against the oracle before any kernel runs it: tests/cpp/fused_model_check.cpp
models the 16-bit half-unit recurrence with its offset and sentinel, the walk
weights built by paths.cpp (build_fused_weights: the stale table's missing and
repeated reverse diagonals, the start-assign restarts at border cells) and the
signed keys of the last pass.  Its disparity maps (WTA + left-right check) must
equal the oracle's for the reference CPU recurrence, the reference GPU one
(second step from C + P1) and the standard one, both tables, 4 and 8 paths,
landscape / portrait / square shapes and D above W."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import oracle
from thundervision_b200 import synthetic

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "thundervision_b200", "csrc")


@pytest.fixture(scope="module")
def model_exe(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("fm") / "fused_model_check")
    subprocess.run(["g++", "-std=c++17", "-O2", "-I/usr/local/cuda/include", "-I" + CSRC,
                    "-I" + os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "fused_model_check.cpp"),
                    os.path.join(CSRC, "paths.cpp"), "-o", exe], check=True)
    return exe


def run_model(exe, tmp, left, right, D, p1, p2, paths, table, sem, lr):
    H, W = left.shape
    src, dst = os.path.join(tmp, "in.bin"), os.path.join(tmp, "out.bin")
    with open(src, "wb") as f:
        f.write(struct.pack("9i", W, H, D, int(2 * p1), int(2 * p2), paths, table, sem, lr))
        f.write(np.ascontiguousarray(left, np.uint8).tobytes())
        f.write(np.ascontiguousarray(right, np.uint8).tobytes())
    r = subprocess.run([exe, src, dst], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    out = np.fromfile(dst, np.uint16)
    return out[:W * H].reshape(H, W), out[W * H:].reshape(H, W)


def oracle_maps(left, right, D, p1, p2, paths, table, sem, lr):
    Lf, Rf = oracle.u8_to_f32(left), oracle.u8_to_f32(right)
    C = oracle.bt_cost(Lf, Rf, D)
    d, _, S = oracle.sgm(C, Lf, p1, p2, paths=paths, table=table, semantics=sem)
    dl, dr = oracle.lr_check(S, d, lr)
    return dl, dr


SHAPES = [(40, 24, 16, 1), (24, 40, 16, 2), (31, 31, 8, 3), (57, 13, 64, 4), (13, 57, 32, 5), (20, 9, 2, 6),
          (96, 64, 64, 7), (64, 96, 100, 8), (3, 2, 16, 9), (17, 2, 8, 10), (2, 17, 8, 11), (1, 5, 3, 12),
          (5, 1, 3, 13), (2, 2, 2, 14), (3, 3, 16, 15)]


@pytest.mark.parametrize("W,H,D,seed", SHAPES)
@pytest.mark.parametrize("sem", [oracle.SEM_REF_CPU, oracle.SEM_STANDARD, oracle.SEM_REF_GPU])
@pytest.mark.parametrize("table", [oracle.TABLE_REF, oracle.TABLE_FULL])
def test_model_equals_oracle(model_exe, tmp_path, W, H, D, seed, sem, table):
    left, right = synthetic.make_pair(W, H, D, seed, n_rects=3)[:2]
    for paths in (8, 4):
        got = run_model(model_exe, str(tmp_path), left, right, D, 10.0, 120.0, paths, table, sem, 1)
        want = oracle_maps(left, right, D, 10.0, 120.0, paths, table, sem, 1)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])


@pytest.mark.parametrize("p1,p2", [(0.0, 0.0), (0.5, 0.5), (30.0, 20.0), (7.5, 300.0), (100.0, 640.0)])
def test_model_penalties_and_noise(model_exe, tmp_path, p1, p2):
    """Uniform noise drives the excluded d = D-1 below the minimum often, so
    path costs go negative; extreme penalties stretch the 16-bit ranges."""
    rng = np.random.default_rng(int(p2 * 10 + p1))
    for (W, H, D) in ((33, 21, 16), (21, 33, 64)):
        left = rng.integers(0, 256, (H, W)).astype(np.uint8)
        right = rng.integers(0, 256, (H, W)).astype(np.uint8)
        got = run_model(model_exe, str(tmp_path), left, right, D, p1, p2, 8, oracle.TABLE_REF,
                        oracle.SEM_REF_CPU, 1)
        want = oracle_maps(left, right, D, p1, p2, 8, oracle.TABLE_REF, oracle.SEM_REF_CPU, 1)
        np.testing.assert_array_equal(got[0], want[0])
        np.testing.assert_array_equal(got[1], want[1])
