"""CPU checks of bench.py's reference arm.

The arm loads nothing but the reference build (oracle/_ref/libdolref.so): its
input volume comes from a numpy restatement of the library's value-noise
generator, and each timed step transforms a bounded sample of every pass of
the full volume.  These tests pin the restatement to the library's host
generator and show that a sample computes the same values as the whole
transform on the lines it covers.
"""
import ctypes as C
import importlib.util
import os

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("dims,spacing,seed", [((64, 48, 40), 16, 3), ((33, 17, 50), 16, 3), ((40, 40, 40), 8, 11)])
def test_noise_restatement_matches_library_generator(bench, dol, O, dims, spacing, seed):
    w, h, d = dims
    words = np.zeros(O.mask_words(w, h, d), np.uint32)
    dol.lib().dol_gen_value_noise_3d_host(w, h, d, spacing, C.c_uint32(seed), words.ctypes.data_as(C.c_void_p))
    want = O.mask_to_bool(words, dims)
    got = np.stack(list(bench.noise_slices(w, h, d, spacing, seed)))
    np.testing.assert_array_equal(got, want)


@pytest.mark.parametrize("fraction", [4, 16])
def test_reference_sample_matches_whole_transform(bench, O, fraction):
    if O.ref() is None:
        pytest.skip("reference build (oracle/_ref) absent")
    n = 64
    rs = bench.ReferenceSample(n, n, n, fraction=fraction, threads=3)
    assert rs.kind == "reference"
    for _ in range(2):   # steps repeat on the same inputs
        rs.step()
    occ = np.stack(list(bench.noise_slices(n, n, n, bench.SPACING, bench.SEED)))
    want = O.sdf_signed_felzenszwalb(O.bool_to_mask(occ), (n, n, n))
    z0, z1 = rs.z0, rs.z0 + rs.nz
    x0, x1 = rs.x0, rs.x0 + rs.nx
    # x rows and the sqrtf difference of the slab: the whole transform's values
    np.testing.assert_array_equal(rs.out.view(np.uint32), want[z0:z1].view(np.uint32))
    # z then y lines of the sampled columns: the slab's after-y field where they meet
    for s in range(2):
        np.testing.assert_array_equal(rs.A[s][z0:z1, :, x0:x1], rs.Y[s][:, :, x0:x1])
    assert rs.voxels * fraction == n ** 3


def test_clock_sampler_reads_nvml_reasons(bench, monkeypatch):
    """The timed region's clock record through NVML (a fake module here):
    samples taken while the region runs, reason bits mapped to their names."""
    import sys
    import time
    import types
    fake = types.ModuleType("pynvml")
    fake.NVML_CLOCK_SM = 1
    fake.nvmlInit = lambda: None
    fake.nvmlShutdown = lambda: None
    fake.nvmlDeviceGetHandleByUUID = lambda u: "h"
    fake.nvmlDeviceGetHandleByIndex = lambda i: "h"
    fake.nvmlDeviceGetMaxClockInfo = lambda h, c: 1965
    fake.nvmlDeviceGetClockInfo = lambda h, c: 1950
    fake.nvmlDeviceGetCurrentClocksEventReasons = lambda h: 0x4 | 0x40
    monkeypatch.setitem(sys.modules, "pynvml", fake)
    c = bench.ClockSampler(0)
    c.start()
    time.sleep(0.03)
    rec = c.stop()
    assert rec["source"] == "nvml" and rec["samples"] > 0
    assert rec["sm_mhz"] == 1950.0 and rec["sm_max_mhz"] == 1965.0
    assert rec["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
