"""The C++ host interface (namespace DOL): compile a small driver against the
shim header and libdol_b200.so like a reference user would, then (GPU) run it
and compare its output with the oracle running the same reference calls."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "distance-occlusion_b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory, dol):
    dol.lib()
    exe = tmp_path_factory.mktemp("shim") / "shim_driver"
    cmd = ["g++", "-O2", "-std=c++17", "-I" + os.path.join(PKG, "shim"), os.path.join(ROOT, "tests", "shim_driver.cpp"),
           "-L" + PKG, "-ldol_b200", "-Wl,-rpath," + PKG, "-o", str(exe)]
    subprocess.run(cmd, check=True)
    return str(exe)


def test_shim_driver_links(driver):
    assert os.path.exists(driver)


@pytest.mark.gpu
@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("sgn", [0, 1])
@pytest.mark.parametrize("dims", [(70, 45, 0), (24, 20, 18)])
def test_shim_matches_oracle(driver, O, tmp_path, method, sgn, dims):
    w, h, d = dims
    out = tmp_path / "out.bin"
    subprocess.run([driver, str(method), str(sgn), str(w), str(h), str(d), "40", "9", str(out)], check=True)
    got = np.fromfile(out, dtype=np.int16)
    shape = (w, h) if d == 0 else (w, h, d)
    m = O.new_mask(*shape)
    O.add_block(m, shape, 4 if d == 0 else 6)
    O.add_points(m, shape, 40, 9)
    start = O.border_init(m, shape) if sgn else O.init_deltas(m, shape)
    want = O.propagate(["danielsson", "fastsweep", "jumpflood"][method], start, shape, 2 if sgn else 1)
    np.testing.assert_array_equal(got, want.reshape(-1))


@pytest.mark.gpu
@pytest.mark.parametrize("dims", [(70, 45), (300, 7)])
def test_shim_chamfer_matches_oracle(driver, O, tmp_path, dims):
    """DOL::InitDistancesFromBitMask(int16) + DOL::Chamfer, as GenerateDistanceChamfer calls them."""
    w, h = dims
    out = tmp_path / "out.bin"
    subprocess.run([driver, "4", "0", str(w), str(h), "0", "40", "9", str(out)], check=True)
    got = np.fromfile(out, dtype=np.int16)
    m = O.new_mask(w, h)
    O.add_block(m, dims, 4)
    O.add_points(m, dims, 40, 9)
    want, mult = O.chamfer(O.init_distances_int(m, dims, np.int16, 32767 - 16), dims)
    assert mult == 3
    np.testing.assert_array_equal(got, want.reshape(-1))
