"""Generate the golden vectors in tests/golden/ from the REFERENCE library.

Runs only where the reference sources were compiled into oracle/_ref/
(`make -C oracle`, which needs the reference checkout).  Every output here
comes from the unmodified reference code (oracle/ref_wrap.cpp includes
DistanceOcclusionLib.cpp as it lies).  Small cases are stored whole
(golden_small.npz); configuration-sized cases as SHA-256 digests of the output
bytes (golden_digests.json), which keeps the fixtures a few hundred KB.

    python tests/golden/gen_golden.py            # small cases, 1024^2 and 64^3 digests
    python tests/golden/gen_golden.py --full     # adds the benchmarked sizes (a few minutes, ~20 GB RAM)
    python tests/golden/gen_golden.py --sparse   # adds 1024^3 volumes of 2000 points and of none

--full digests the reference's outputs on the two benchmarked volumes, from
the same synthetic masks the library generates (its host generator; the
mask digests pin host and device generation to each other):
  1024^3 value noise (lattice 16, seed 3): signed Felzenszwalb SDF (the
      reference's 1D routine along z, y, x for each sign, sqrt, difference)
      and signed Danielsson deltas (border init, cw = 2);
  256^3, 32 boxes + 32 spheres (sides / radii 4-40, seed 7): border init,
      Danielsson / FastSweep / JumpFlood with cw = 2, signed Felzenszwalb SDF.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402


def rand_mask(rng, dims, p):
    return O.bool_to_mask(rng.random(tuple(reversed(dims))) < p)


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    if O.ref() is None:
        raise SystemExit("oracle/_ref/libdolref.so missing: build it with `make -C oracle` next to the reference")
    rng = np.random.default_rng(20261203)
    small = {}
    cases2 = [("r2a", (64, 48), 0.08), ("r2b", (33, 17), 0.3), ("r2c", (97, 5), 0.5), ("r2d", (40, 40), 0.0)]
    for name, dims, p in cases2:
        m = rand_mask(rng, dims, p)
        small[f"{name}_mask"] = m
        small[f"{name}_dims"] = np.array(dims)
        ini = O.init_deltas(m, dims, use_ref=True)
        bor = O.border_init(m, dims, use_ref=True)
        small[f"{name}_init"] = ini
        small[f"{name}_init_inv"] = O.init_deltas(m, dims, True, use_ref=True)
        small[f"{name}_border"] = bor
        for meth in ("danielsson", "fastsweep", "jumpflood"):
            small[f"{name}_{meth}_cw1"] = O.propagate(meth, ini, dims, 1, use_ref=True)
            small[f"{name}_{meth}_cw2"] = O.propagate(meth, bor, dims, 2, use_ref=True)
        small[f"{name}_bruteforce_cw1"] = O.propagate("bruteforce", ini, dims, 1, use_ref=True)
        small[f"{name}_bruteforce_cw2"] = O.propagate("bruteforce", bor, dims, 2, use_ref=True)
        f = O.init_distances(m, dims, use_ref=True)
        small[f"{name}_felz"] = O.felzenszwalb(f, dims, use_ref=True)
    cases3 = [("r3a", (20, 12, 9), 0.1), ("r3b", (33, 7, 6), 0.4), ("r3c", (16, 16, 16), 0.02)]
    for name, dims, p in cases3:
        m = rand_mask(rng, dims, p)
        small[f"{name}_mask"] = m
        small[f"{name}_dims"] = np.array(dims)
        ini = O.init_deltas(m, dims, use_ref=True)
        bor = O.border_init(m, dims, use_ref=True)
        small[f"{name}_init"] = ini
        small[f"{name}_border"] = bor
        for meth in ("danielsson", "fastsweep", "jumpflood"):
            small[f"{name}_{meth}_cw1"] = O.propagate(meth, ini, dims, 1, use_ref=True)
            small[f"{name}_{meth}_cw2"] = O.propagate(meth, bor, dims, 2, use_ref=True)
        small[f"{name}_bruteforce_cw1"] = O.propagate("bruteforce", ini, dims, 1, use_ref=True)
        big = np.float32(np.finfo(np.float32).max)
        f = np.where(O.mask_to_bool(m, dims), np.float32(0), big).astype(np.float32)
        small[f"{name}_felz"] = O.felzenszwalb(f, dims, use_ref=True, threads=1)
    np.savez_compressed(os.path.join(HERE, "golden_small.npz"), **small)

    dig = {}
    # configuration 1: 1024x1024, 100 points, seed 1 (BitMaskAddPoints), unsigned
    dims = (1024, 1024)
    m = O.add_points(O.new_mask(*dims), dims, 100, 1, use_ref=True)
    dig["c1_mask"] = digest(m)
    ini = O.init_deltas(m, dims, use_ref=True)
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        dig[f"c1_{meth}_cw1"] = digest(O.propagate(meth, ini, dims, 1, use_ref=True))
    bor = O.border_init(m, dims, use_ref=True)
    dig["c1_border"] = digest(bor)
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        dig[f"c1_{meth}_cw2"] = digest(O.propagate(meth, bor, dims, 2, use_ref=True))
    dig["c1_felz"] = digest(O.felzenszwalb(O.init_distances(m, dims, use_ref=True), dims, use_ref=True))
    # 3D: 64^3 with a 6-sided test box plus 200 points (seed 12345)
    dims = (64, 64, 64)
    m = O.add_block(O.new_mask(*dims), dims, 6, use_ref=True)
    m = O.add_points(m, dims, 200, 12345, use_ref=True)
    dig["v64_mask"] = digest(m)
    bor = O.border_init(m, dims, use_ref=True)
    dig["v64_border"] = digest(bor)
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        dig[f"v64_{meth}_cw2"] = digest(O.propagate(meth, bor, dims, 2, use_ref=True))
    ini = O.init_deltas(m, dims, use_ref=True)
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        dig[f"v64_{meth}_cw1"] = digest(O.propagate(meth, ini, dims, 1, use_ref=True))
    with open(os.path.join(HERE, "golden_digests.json")) as f:
        old = json.load(f)
    kept = ("s3_",) if "--full" in sys.argv else ("c2_", "c3_", "s3_")
    if "--sparse" in sys.argv:
        kept = tuple(k for k in kept if k != "s3_")
    dig.update({k: v for k, v in old.items() if k.startswith(kept)})
    if "--full" in sys.argv:
        dig.update(full_size())
    if "--sparse" in sys.argv:
        dig.update(sparse_size())
    with open(os.path.join(HERE, "golden_digests.json"), "w") as f:
        json.dump(dig, f, indent=1, sort_keys=True)
    print("wrote", len(small), "arrays and", len(dig), "digests")


def _signed_felz_ref(m, dims, threads):
    b = O.mask_to_bool(m, dims)
    big = np.float32(np.finfo(np.float32).max)
    e_occ = O.felzenszwalb(np.where(b, np.float32(0), big).astype(np.float32), dims, use_ref=True, threads=threads)
    e_emp = O.felzenszwalb(np.where(b, big, np.float32(0)).astype(np.float32), dims, use_ref=True, threads=threads)
    del b
    return (np.sqrt(e_occ) - np.sqrt(e_emp)).astype(np.float32)


def full_size():
    import ctypes as C
    sys.path.insert(0, ROOT)
    import bench
    L = bench.load_dol().lib()
    threads = os.cpu_count() or 1
    dig = {}
    # 256^3 shapes
    n = 256
    dims = (n, n, n)
    m = np.zeros(O.mask_words(*dims), np.uint32)
    L.dol_gen_shapes_3d_host(n, n, n, 32, 32, 4, 40, C.c_uint32(7), m.ctypes.data_as(C.c_void_p))
    dig["c2_mask"] = digest(m)
    bor = O.border_init(m, dims, use_ref=True)
    dig["c2_border"] = digest(bor)
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        dig[f"c2_{meth}_cw2"] = digest(O.propagate(meth, bor, dims, 2, use_ref=True))
        print("c2", meth, flush=True)
    dig["c2_felz_signed"] = digest(_signed_felz_ref(m, dims, threads))
    # 1024^3 value noise
    n = 1024
    dims = (n, n, n)
    m = np.zeros(O.mask_words(*dims), np.uint32)
    L.dol_gen_value_noise_3d_host(n, n, n, 16, C.c_uint32(3), m.ctypes.data_as(C.c_void_p))
    dig["c3_mask"] = digest(m)
    dig["c3_felz_signed"] = digest(_signed_felz_ref(m, dims, threads))
    print("c3 felzenszwalb", flush=True)
    bor = O.border_init(m, dims, use_ref=True)
    dig["c3_danielsson_cw2"] = digest(O.propagate("danielsson", bor, dims, 2, use_ref=True))
    print("c3 danielsson", flush=True)
    return dig


def sparse_size():
    """The reference's signed Felzenszwalb where the other state is far away:
    1024^3 with 2000 set voxels (BitMaskAddPoints, seed 1) and 1024^3 with none."""
    threads = os.cpu_count() or 1
    dig = {}
    n = 1024
    dims = (n, n, n)
    m = O.add_points(np.zeros(O.mask_words(*dims), np.uint32), dims, 2000, 1, use_ref=True)
    dig["s3_points2000_mask"] = digest(m)
    dig["s3_points2000_felz_signed"] = digest(_signed_felz_ref(m, dims, threads))
    print("s3 points", flush=True)
    m = np.zeros(O.mask_words(*dims), np.uint32)
    dig["s3_empty_felz_signed"] = digest(_signed_felz_ref(m, dims, threads))
    print("s3 empty", flush=True)
    return dig


if __name__ == "__main__":
    main()
