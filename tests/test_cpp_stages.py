"""The C++ stage classes (include/tdv_stages.hpp) -- host code shaped like
LibThunderVision's stage plugins (tdvision/matchingcost.hpp:48-49,
tdvision/optimizer.hpp:46) -- compiled with g++ against libtdvb200.so.

CPU: the header compiles and bad arguments throw CUException with the ABI's
status before any CUDA call (the matcher stages, the rectifier, the dilation
and the PLY exporter).  GPU: the stage chains give the oracle's maps on
the same pair (REF_CPU / REF_GPU SGM with the reference's table, P2 adjusted
by the intensity step, BT cost in [0,1] intensities; DP; FastWTA; the fused
Lab-style matcher).
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from thundervision_b200 import _lib as L
from thundervision_b200 import synthetic as syn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CUDA = "/usr/local/cuda"


def build_demo(out):
    """Compiles tests/cpp/stages_demo.cpp against libtdvb200.so into `out`."""
    L.build()
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    libdir = os.path.dirname(L.LIB_PATH)
    cmd = ["g++", "-std=c++17", "-O1", "-I" + os.path.join(ROOT, "include"), "-I" + CUDA + "/include",
           os.path.join(ROOT, "tests", "cpp", "stages_demo.cpp"), "-L" + libdir, "-ltdvb200",
           "-L" + CUDA + "/lib64", "-lcudart", "-Wl,-rpath," + libdir, "-Wl,-rpath," + CUDA + "/lib64",
           "-o", out]
    subprocess.run(cmd, check=True)
    return out


@pytest.fixture(scope="module")
def demo(tmp_path_factory):
    return build_demo(str(tmp_path_factory.mktemp("cpp") / "stages_demo"))


def test_stage_classes_validate_before_cuda(demo):
    r = subprocess.run([demo, "validate"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert "validate: ok" in r.stdout


@pytest.mark.gpu
def test_stage_chains_match_oracle(demo, orc, tmp_path):
    W, H, D = 96, 64, 16
    Lh, Rh, _, _ = syn.make_pair(W, H, D, 21, n_rects=4)
    lp, rp = tmp_path / "l.u8", tmp_path / "r.u8"
    Lh.tofile(lp)
    Rh.tofile(rp)
    prefix = str(tmp_path / "out")
    r = subprocess.run([demo, "run", str(W), str(H), str(D), str(lp), str(rp), prefix],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {k: np.fromfile(f"{prefix}.{k}.u16", dtype=np.uint16).reshape(H, W)
           for k in ("sgm_ref_cpu", "sgm_ref_gpu", "sgm_filtered", "dp", "fastwta", "lab")}

    Lf = orc.u8_to_f32(Lh, 1.0 / 255.0)
    Rf = orc.u8_to_f32(Rh, 1.0 / 255.0)
    C = orc.bt_cost(Lf, Rf, D, layout=orc.LAYOUT_REF_WHD)
    for key, sem in (("sgm_ref_cpu", orc.SEM_REF_CPU), ("sgm_ref_gpu", orc.SEM_REF_GPU)):
        d_ref, _, _ = orc.sgm(C, Lf, 30.0 / 255.0, 150.0 / 255.0, p2_mode=orc.P2_ADJUST, table=orc.TABLE_REF,
                              semantics=sem, layout=orc.LAYOUT_REF_WHD, want_S=False)
        np.testing.assert_array_equal(got[key], d_ref, err_msg=key)
    from oracle import image_ops as io
    Gl, Gr = io.gauss5(Lf), io.gauss5(Rf)
    Cg = orc.bt_cost(Gl, Gr, D, layout=orc.LAYOUT_REF_WHD)
    d_ref, _, _ = orc.sgm(Cg, Gl, 30.0 / 255.0, 150.0 / 255.0, p2_mode=orc.P2_ADJUST, table=orc.TABLE_REF,
                          semantics=orc.SEM_REF_GPU, layout=orc.LAYOUT_REF_WHD, want_S=False)
    np.testing.assert_array_equal(got["sgm_filtered"], d_ref)
    d_ref, _ = orc.dp(C, layout=orc.LAYOUT_REF_WHD)
    np.testing.assert_array_equal(got["dp"], d_ref)
    d_ref, _ = orc.fastwta(Lf, Rf, D, radius=3)
    np.testing.assert_array_equal(got["fastwta"], d_ref)
    L8, R8 = orc.u8_to_f32(Lh), orc.u8_to_f32(Rh)
    d_ref, _, _ = orc.sgm(orc.bt_cost(L8, R8, D), L8, 10.0, 120.0, want_S=False)
    np.testing.assert_array_equal(got["lab"], d_ref)
