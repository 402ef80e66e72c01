"""The reference's own caller, unmodified, on the B200 library.

oracle/Makefile (target `tool`) compiles the reference's command-line tool
(DistanceOcclusionTool.cpp, which reaches the library through FindDeltas,
DistanceOcclusionTool.cpp:711-739 / :937-965, and the other Generate* paths)
twice from the same sources: distocc_ref with the reference library, as the
reference's Makefile does, and distocc_b200 with tool_ref_half.cpp (the
reference library minus every function the B200 library provides) and
libdol_b200.so.  The CPU test checks the link: in distocc_b200 the distance
functions and the occlusion sweeps are undefined, to be bound to
libdol_b200.so at load time, while BruteForce and the shadow sweep stay
defined from the reference.  The
GPU test runs both tools on the same command lines and compares every image
they write, byte for byte.
"""
import filecmp
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
TOOL_REF = os.path.join(REF, "distocc_ref")
TOOL_B200 = os.path.join(REF, "distocc_b200")

GPU_SIDE = ["InitDistancesFromBitMask", "Chamfer", "Felzenszwalb", "InitDeltasFromBitMask",
            "InitBorderDeltasFromBitMask", "FastSweep", "Danielsson", "JumpFlood", "InitDirWFromBitMask",
            "OcclusionSweep"]
REF_SIDE = ["BruteForce", "ShadowSweep"]


def _need_tools():
    if not (os.path.exists(TOOL_REF) and os.path.exists(TOOL_B200)):
        pytest.skip("tool builds absent (make -C oracle tool needs the reference sources)")


def test_tool_links_distance_functions_to_the_library():
    _need_tools()
    if shutil.which("nm") is None:
        pytest.skip("nm not available")
    syms = subprocess.run(["nm", "-C", TOOL_B200], capture_output=True, text=True, check=True).stdout.splitlines()
    kind = {}
    for ln in syms:
        parts = ln.split(None, 2) if not ln.startswith(" ") else ["", *ln.split(None, 1)]
        if len(parts) == 3 and parts[2].startswith("DOL::"):
            name = parts[2][5:].split("(")[0]
            kind.setdefault(name, set()).add(parts[1])
    for name in GPU_SIDE:
        assert kind.get(name) == {"U"}, f"DOL::{name} should come from libdol_b200.so, nm says {kind.get(name)}"
    for name in REF_SIDE:
        assert "T" in kind.get(name, set()), f"DOL::{name} should be the reference's, nm says {kind.get(name)}"
    ldd = subprocess.run(["ldd", TOOL_B200], capture_output=True, text=True).stdout
    assert "libdol_b200.so" in ldd and "not found" not in ldd.split("libdol_b200.so")[1].splitlines()[0]


# command lines: unsigned (-d), single-pass signed (-s), two-pass signed (-S),
# images and volumes, every delta method, Chamfer and Felzenszwalb, image
# inputs, output variants, the BruteForce checks (-c) and occlusion (-x)
COMMANDS = [
    "-d -w 1024 -p 100 1",
    "-d -w 1024 -p 100 1 -m 1",
    "-d -w 1024 -p 100 1 -m 2",
    "-d -w 1024 -p 100 1 -m 4",
    "-d -w 1024 -p 100 1 -m 5",
    "-d -w 200 150 -p 30 9 -c",
    "-s -w 512 -b 4 -p 50 7",
    "-s -w 512 -b 4 -p 50 7 -m 1 -i 1",
    "-s -w 333 257 -p 60 5 -m 2 -i 2",
    "-S -w 300 200 -p 40 3",
    "-S -w 300 200 -p 40 3 -m 1 -i 2",
    "-S -w 300 200 -p 40 3 -m 2",
    "-s -f tiger.png",
    "-s -f kiwi.png -i 2",
    "-S -f tiger.png -m 2",
    "-d -W 48 40 32 -p 30",
    "-d -W 48 40 32 -p 30 -m 1",
    "-d -W 48 40 32 -p 30 -m 2",
    "-s -W 64 -b 6 -p 200",
    "-s -W 64 -b 6 -p 200 -m 1",
    "-s -W 64 -b 6 -p 200 -m 2 -i 1",
    "-S -W 40 -p 20 -m 0",
    "-s -W 24 20 16 -p 10 -c",
    "-x -w 128 -p 20",
    "-x -w 300 200 -b 4 -p 30 5 -m 2",
    "-x -W 32 -p 20",
    "-x -W 40 30 20 -b 6 -p 30 -m 1",
    "-x -W 24 -p 10 -m 2",
]


@pytest.mark.gpu
@pytest.mark.parametrize("cmd", COMMANDS)
def test_tool_outputs_identical(cuda, tmp_path, cmd):
    _need_tools()
    outs = {}
    for tag, exe in (("ref", TOOL_REF), ("b200", TOOL_B200)):
        d = tmp_path / tag
        d.mkdir()
        args = cmd.split()
        args = [os.path.join(REF, a) if a.endswith(".png") else a for a in args]
        r = subprocess.run([exe, *args, "-o", str(d / "out")], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, f"{tag}: {cmd}\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}"
        outs[tag] = sorted(os.listdir(d))
    assert outs["ref"] and outs["ref"] == outs["b200"], (outs["ref"][:5], outs["b200"][:5])
    diff = [f for f in outs["ref"] if not filecmp.cmp(tmp_path / "ref" / f, tmp_path / "b200" / f, shallow=False)]
    assert not diff, f"{len(diff)} of {len(outs['ref'])} images differ, e.g. {diff[:3]}"
