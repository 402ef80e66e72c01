"""Benchmark: signed distance field of a 1024^3 volume on one B200 per rank.

Workload (the large 3D SDF throughput case): a 1024^3 1-bit volume of 3D value
noise (lattice spacing 16, uniform lattice values from the reference's LCG,
seed 3, trilinear, thresholded at 1/2, ~50% occupied).  One step = the
mask-driven exact Felzenszwalb transform producing the signed float field
(distance to set voxels minus distance to clear voxels) from a device-resident
mask.  Metric: Gvoxels/s of the whole job.  Inputs and outputs (128 MiB mask,
4 GiB field) are far larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dol|reference]

--impl reference times the reference's own CPU code for the same output on the
same 1024^3 volume (the reference's 1D Felzenszwalb routine applied along z,
y, x -- it has no 3D driver -- twice, for the two signs, then sqrtf and the
difference, on all host cores); each step is a bounded sample, 1/16 of every
pass, run with the full volume's strides on the real intermediate fields.
Under torchrun each rank runs an independent replica (the transform needs the
whole volume; there is no exchange step), timed on the device, max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
SIDE = 1024          # volume side; --side changes it (profiling runs use a smaller case)
W = H = D = SIDE
SPACING, SEED = 16, 3
METRIC = "SDF Gvoxels/s (1024^3 value-noise volume, signed Felzenszwalb EDT, mask -> f32)"
WORKLOAD = "1024^3 value noise (lattice 16, seed 3, threshold 1/2), signed Felzenszwalb SDF, f32 out"
# algorithmic bytes per voxel of each kernel of the transform
PASS_BYTES = {"edt_x": 1 / 8 + 2, "edt_y": 2 + 4, "edt_z_final": 4 + 4}


def load_dol():
    pkg = os.path.join(ROOT, "distance-occlusion_b200")
    spec = importlib.util.spec_from_file_location("dol_b200", os.path.join(pkg, "__init__.py"),
                                                  submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dol_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    queries (read only) from a thread every 2 ms, else nvidia-smi, whose
    samples count from the first one after its start-up."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    BITS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
            ("sw_power_cap", 0x4))

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []
        self.samples = []
        self.nvml = None
        self.n0 = 0

    def _start_nvml(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            try:
                import torch
                u = str(torch.cuda.get_device_properties(self.idx).uuid)
                h = pynvml.nvmlDeviceGetHandleByUUID(u if u.startswith("GPU-") else "GPU-" + u)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(self.idx)
            reasons = (getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or
                       pynvml.nvmlDeviceGetCurrentClocksThrottleReasons)
            mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
            pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
            reasons(h)
        except Exception:
            return False
        self.nvml = pynvml
        self.stop_ev = threading.Event()

        def loop():
            while not self.stop_ev.is_set():
                try:
                    self.samples.append((float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)), mx,
                                         int(reasons(h))))
                except Exception:
                    break
                self.stop_ev.wait(0.002)

        self.t = threading.Thread(target=loop, daemon=True)
        self.t.start()
        return True

    def start(self):
        if self._start_nvml():
            return
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "10"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.lines and time.time() - t0 < 3.0 and self.proc.poll() is None:
                time.sleep(0.005)
            self.n0 = len(self.lines)
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_ev.set()
            self.t.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
            sm = [x[0] for x in self.samples]
            reasons = sorted({n for _, _, r in self.samples for n, bit in self.BITS if r & bit})
            return {"sm_mhz": float(np.median(sm)) if sm else None,
                    "sm_max_mhz": max(x[1] for x in self.samples) if sm else None,
                    "reasons": reasons, "samples": len(sm), "source": "nvml"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = [n for n, _ in self.BITS]
        lines = self.lines[self.n0:] or self.lines[-1:]   # none inside a short region: the next one
        for ln in lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi"}


def max_over_ranks(x, pg, device="cuda"):
    """The slowest rank's value; every rank calls it (a no-op on one rank)."""
    if not pg:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_gvox_per_s(world, voxels_per_rank, seconds):
    """Whole-job throughput of `world` independent replicas timed at `seconds` (max over ranks)."""
    return world * voxels_per_rank / seconds / 1e9


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- reference arm ----
# The reference's CPU code for the same output: its 1D Felzenszwalb routine
# (DistanceOcclusionLib.cpp:1026-1062) applied along z, y and x (it has no 3D
# driver) to the two transforms of the signed field, then sqrtf and the
# difference.  Only oracle/_ref/libdolref.so (the reference compiled from its
# own sources) is loaded; the input volume comes from a numpy restatement of
# the generator, so nothing of this library runs in that arm.

REF_FRACTION = 16    # a step transforms 1/16 of every pass's lines (the whole 1024^3 takes ~20 s)


def noise_lattice(w, h, d, L, seed):
    """Lattice values of the value-noise volume: (d//L+2, h//L+2, w//L+2)
    uint16 from the reference's LCG (DistanceOcclusionLib.cpp:28-32), x fastest."""
    gx, gy, gz = w // L + 2, h // L + 2, d // L + 2
    vals = np.empty(gx * gy * gz, np.int64)
    s = seed & 0xFFFFFFFF
    for i in range(vals.size):
        s = (s * 1103515245 + 12345) & 0xFFFFFFFF
        vals[i] = (s * 65536) >> 32
    return vals.reshape(gz, gy, gx)


def noise_slices(w, h, d, L, seed):
    """Yields bool[h, w] occupancy per slice z of the value-noise volume: set
    iff sum(v * wx * wy * wz) over the 8 lattice corners >= 32768 * L^3, the
    integer form of "trilinear value >= 1/2" (the library's generator)."""
    lat = noise_lattice(w, h, d, L, seed)
    xs, ys = np.arange(w), np.arange(h)
    i, fx = xs // L, xs % L
    j, fy = ys // L, ys % L
    wx0, wx1 = (L - fx)[None, :], fx[None, :]
    wy0, wy1 = (L - fy)[:, None], fy[:, None]
    thr = 32768 * L ** 3
    planes = {}

    def plane(k):   # bilinear weights applied within lattice plane k, int64[h, w]
        if k not in planes:
            if len(planes) >= 2:
                del planes[min(planes)]   # slices advance in z: the lowest plane is done
            v = lat[k]
            r0 = wx0 * v[np.ix_(j, i)] + wx1 * v[np.ix_(j, i + 1)]
            r1 = wx0 * v[np.ix_(j + 1, i)] + wx1 * v[np.ix_(j + 1, i + 1)]
            planes[k] = wy0 * r0 + wy1 * r1
        return planes[k]

    for z in range(d):
        k, fz = divmod(z, L)
        yield ((L - fz) * plane(k) + fz * plane(k + 1)) >= thr


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class ReferenceSample:
    """Bounded samples of the reference's signed Felzenszwalb on the w x h x d
    value-noise volume.  Untimed set-up: the volume, the two 0 / FLT_MAX
    inputs, the full z pass (A) and the y pass of one slab of d/f slices (Y).
    A timed step then runs, with the full volume's strides and on the real
    intermediate fields, 1/f of every pass: z lines of w/f columns (raw -> A),
    the y lines of those columns (A -> A), the x rows of the slab (Y -> X),
    and sqrtf(occ) - sqrtf(emp) over the slab: 1/f of the whole transform."""

    def __init__(self, w, h, d, fraction=REF_FRACTION, threads=None):
        self.threads = threads or host_threads()
        here = os.path.join(ROOT, "oracle")
        ref_path = os.path.join(here, "_ref", "libdolref.so")
        if os.path.exists(ref_path):
            self.kind, self.L = "reference", C.CDLL(ref_path)
        else:   # the oracle's restatement of the same routine, one thread
            self.kind, self.L = "port", C.CDLL(os.path.join(here, "liboracle.so"))
            self.threads = 1
        self.w, self.h, self.d = w, h, d
        f = max(1, min(fraction, w, d))
        self.nx, self.nz = w // f, d // f
        self.x0, self.z0 = (w - self.nx) // 2, (d - self.nz) // 2
        self.voxels = self.nx * h * d          # voxels of one pass's sample (equal for all three)
        self.fraction = w * h * d / self.voxels
        big = np.float32(np.finfo(np.float32).max)
        self.raw = [np.empty((d, h, w), np.float32) for _ in range(2)]
        for z, occ in enumerate(noise_slices(w, h, d, SPACING, SEED)):
            self.raw[0][z] = np.where(occ, np.float32(0), big)   # transform to set voxels
            self.raw[1][z] = np.where(occ, big, np.float32(0))   # transform to clear voxels
        self.A = [np.empty_like(r) for r in self.raw]
        z0, z1 = self.z0, self.z0 + self.nz
        for s in range(2):
            self._pass(self.raw[s], self.A[s], 0, 0, h, 0, w)        # full z pass
            self._pass(self.A[s], self.A[s], 1, z0, z1, 0, w)        # y pass of the slab
        self.Y = [np.ascontiguousarray(a[z0:z1]) for a in self.A]
        self.X = [np.empty_like(y) for y in self.Y]
        self.out = np.empty_like(self.Y[0])
        self.sample = (f"1/{self.fraction:.0f} of every pass per step on the {w}x{h}x{d} volume "
                       f"(z and y lines of x in [{self.x0},{self.x0 + self.nx}), x rows of z in [{z0},{z1})), "
                       f"both transforms, with the reference's 1D Felzenszwalb (DistanceOcclusionLib.cpp:1026-1062), "
                       f"then sqrtf difference; {self.threads} host threads")

    def _pass(self, src, dst, pas, a0, a1, b0, b1, dims=None):
        w, h, d = dims or (self.w, self.h, self.d)
        vp = lambda a: a.ctypes.data_as(C.c_void_p)
        if self.kind == "reference":
            self.L.ref_felzenszwalb_3d_pass(w, h, d, vp(src), vp(dst), pas, a0, a1, b0, b1, self.threads)
        else:
            n = max(w, h, d)
            v, zz, line = np.empty(n, np.int32), np.empty(n + 1, np.float32), np.empty(n, np.float32)
            self.L.dolo_felzenszwalb_3d_pass(w, h, d, vp(src), vp(dst), pas, a0, a1, b0, b1, vp(v), vp(zz), vp(line))

    def step(self):
        """One timed sample; returns its seconds."""
        w, h, d = self.w, self.h, self.d
        xb = (self.x0, self.x0 + self.nx)
        t = time.perf_counter()
        for s in range(2):
            self._pass(self.raw[s], self.A[s], 0, 0, h, *xb)                     # z lines
        for s in range(2):
            self._pass(self.A[s], self.A[s], 1, 0, d, *xb)                       # y lines
        for s in range(2):
            self._pass(self.Y[s], self.X[s], 2, 0, self.nz, 0, h, (w, h, self.nz))   # x rows
        n = self.out.size
        if self.kind == "reference":
            self.L.ref_sqrt_diff(C.c_longlong(n), self.X[0].ctypes.data_as(C.c_void_p),
                                 self.X[1].ctypes.data_as(C.c_void_p), self.out.ctypes.data_as(C.c_void_p),
                                 self.threads)
        else:
            np.subtract(np.sqrt(self.X[0]), np.sqrt(self.X[1]), out=self.out)
        return time.perf_counter() - t


def cpu_reference_sample(steps=3, warmup=1):
    """The reference arm's measurement as the cpu_baseline of a GPU run: a few
    steps of ReferenceSample on the benchmarked volume.  Returns the
    cpu_baseline object (Gvox/s of the whole transform)."""
    rs = ReferenceSample(W, H, D)
    for _ in range(warmup):
        rs.step()
    t = [rs.step() for _ in range(steps)]
    value = rs.voxels / float(np.mean(t)) / 1e9
    return {"value": value, "unit": "Gvoxels/s", "cores": rs.threads, "kind": rs.kind,
            "sample": rs.sample + f"; {steps} timed steps after {warmup} warm-up"}


def bench_config(ws):
    """The benchmarked configuration, identical in both arms."""
    return {"workload": WORKLOAD, "voxels_per_gpu": W * H * D, "parallelism": f"replicas x{ws}",
            "l2": "inputs and outputs > L2 (128 MiB mask in, 4 GiB field out); no flush needed"}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return
    rs = ReferenceSample(W, H, D)
    for _ in range(args.warmup):
        rs.step()
    t_per = [rs.step() for _ in range(args.steps)]
    ms = float(np.mean(t_per)) * 1e3
    value = rs.voxels / (ms * 1e-3) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gvoxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(ws),
        "cpu_baseline": {"value": value, "unit": "Gvoxels/s", "cores": rs.threads, "kind": rs.kind,
                         "sample": rs.sample},
        "e2e": {"value": value, "unit": "Gvoxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- per-configuration lines ----

def _ev_ms(torch, fn, reps=1):
    st = torch.cuda.current_stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(reps):
        fn()
    b.record(st)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def measure_configs(dol, torch, cpu=True, big=True, only=None):
    """Secondary measurements on the other workloads: the 2D default
    (1024^2, 100 points, seed 1, unsigned Danielsson), the 256^3 signed volume
    (32 boxes + 32 spheres, sizes 4-40, seed 7) with every method, the batch
    of 4096 uneven masks + 64 volumes (batched launch vs per-item loop),
    Danielsson on the 1024^3 noise volume, the mask EDT where the other state
    is far (a sparse 2D image, 1024^3 volumes of 2000 points and of none), and
    the occlusion sweeps and mesh voxeliser.  GPU times are CUDA events on
    device-resident data; CPU times are the reference library (oracle/_ref),
    one thread, on the same inputs."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    L = dol.lib()
    sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    res = {}
    ref = O.ref() if cpu else None
    want = (lambda key: only is None or key in only)
    # launch configurations chosen by the library's autotuner (untimed)
    tuned = {}
    for name, kind, shape in (("danielsson_2d", 0, (1024, 1024, 1)), ("danielsson_3d", 1, (256, 256, 256)),
                              ("fastsweep_3d", 3, (256, 256, 256)), ("jumpflood_3d", 5, (256, 256, 256)),
                              ("batch", 6, (1024, 1, 1)), ("edt", 7, (1024, 1024, 1024))):
        if L.dol_autotune(kind, *shape, sp) == 0:
            tuned[name] = L.dol_tune_get(kind, shape[0])
    res["autotuned"] = tuned

    if want("c1"):
        _config1(dol, torch, O, ref, res, (1024, 1024))
    if want("c2"):
        _config2(dol, torch, O, ref, res, L, sp)
    if want("c4"):
        _config4(dol, torch, res, L, sp)
    if want("c5"):
        _config5(dol, torch, res)
    if big and want("c3"):
        _config3(dol, torch, res, L, sp)
    if want("c7"):
        _config_sparse(dol, torch, O, ref, res, L, sp, big)
    if want("c8"):
        _config_occlusion_voxel(dol, torch, O, ref, res)
    if only is not None and "c6" in only:
        _sweep_variants(dol, torch, res, L, sp, big)
    return res


def _sweep_variants(dol, torch, res, L, sp, big=True):
    """Danielsson time per launch configuration of the block schedule (rows
    per block, slices per block, cells per thread) and of the serial engine,
    on the 2D default image, a 256^3 shape volume and the 1024^3 noise
    volume."""
    out = {}
    ROWS, SLICES, DAN2, DAN3 = 8, 9, 0, 1
    dims2 = (1024, 1024)
    m2 = dol.add_points(np.zeros(dol.mask_words(*dims2), np.uint32), dims2, 100, 1)
    md2 = torch.from_numpy(m2.view(np.int32)).cuda()
    base2 = dol.init_deltas(md2, dims2)
    work2 = base2.clone()

    def timed(work, base, dims, cw, reps=1):
        def run():
            work.copy_(base)
            dol.danielsson(work, dims, cw)
        run()
        return _ev_ms(torch, run, reps) - _ev_ms(torch, lambda: work.copy_(base), reps)

    for rows in (8, 16, 32, 64, 128, 65536):
        L.dol_tune_set(ROWS, 1024, rows)
        out[f"2d_1024_rows{rows}_ms"] = timed(work2, base2, dims2, 1, 3)
    L.dol_tune_set(ROWS, 1024, 0)

    n = 256
    dims3 = (n, n, n)
    md3 = torch.empty(dol.mask_words(*dims3), dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_shapes_3d(n, n, n, 32, 32, 4, 40, C.c_uint32(7), C.c_void_p(md3.data_ptr()), sp))
    base3 = dol.init_border(md3, dims3)
    work3 = base3.clone()
    for rows in (4, 8, 16, 32):
        L.dol_tune_set(ROWS, n, rows)
        for z in (2, 4, 8, 16, 0):
            L.dol_tune_set(SLICES, n, z)
            out[f"3d_256_rows{rows}_slices{z or 'auto'}_ms"] = timed(work3, base3, dims3, 2)
    L.dol_tune_set(ROWS, n, 0)
    L.dol_tune_set(SLICES, n, 0)
    for s_ in (1, 2, 4):
        L.dol_tune_set(DAN3, n, s_)
        out[f"3d_256_auto_s{s_}_ms"] = timed(work3, base3, dims3, 2)
    L.dol_tune_set(DAN3, n, 0)
    del work3, base3
    if big:
        side = 1024
        mdv = torch.empty(dol.mask_words(side, side, side), dtype=torch.int32, device="cuda")
        dol.check(L.dol_gen_value_noise_3d(side, side, side, SPACING, C.c_uint32(SEED), C.c_void_p(mdv.data_ptr()), sp))
        dv = torch.empty((side, side, side, 3), dtype=torch.int16, device="cuda")
        for rows, z, s_ in ((8, 0, 0), (8, 32, 0), (8, 64, 0), (16, 32, 0), (8, 32, 2), (8, 32, 8), (16, 32, 8)):
            L.dol_tune_set(ROWS, side, rows)
            L.dol_tune_set(SLICES, side, z)
            L.dol_tune_set(DAN3, side, s_)
            dol.init_border(mdv, (side,) * 3, out=dv)
            torch.cuda.synchronize()
            out[f"3d_1024_rows{rows}_slices{z or 'auto'}_s{s_ or 'auto'}_ms"] = \
                _ev_ms(torch, lambda: dol.danielsson(dv, (side,) * 3, 2), 1)
        L.dol_tune_set(ROWS, side, 0)
        L.dol_tune_set(SLICES, side, 0)
        L.dol_tune_set(DAN3, side, 0)
        del dv, mdv
    res["danielsson_variants"] = out


def _config1(dol, torch, O, ref, res, dims):
    m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
    md = torch.from_numpy(m.view(np.int32)).cuda()
    dl = dol.init_deltas(md, dims)
    base = dl.clone()
    dol.danielsson(dl, dims, 1)
    torch.cuda.synchronize()

    def run_c1():
        dl.copy_(base)
        dol.danielsson(dl, dims, 1)
    t_copy = _ev_ms(torch, lambda: dl.copy_(base), 5)
    t = _ev_ms(torch, run_c1, 5) - t_copy
    c1 = {"workload": "1024^2, 100 points (seed 1), unsigned Danielsson deltas", "gpu_ms": t,
          "gpu_mcells_per_s": 1024 * 1024 / t / 1e3}
    if ref is not None:
        ini = O.init_deltas(m, dims, use_ref=True)
        t0 = time.perf_counter()
        O.propagate("danielsson", ini, dims, 1, use_ref=True)
        c1["cpu_ref_ms"] = (time.perf_counter() - t0) * 1e3
    res["danielsson_2d_1024"] = c1
    # Chamfer 3-4 on the same image, as the tool's GenerateDistanceChamfer (int16, INT16_MAX - 16)
    f0 = dol.init_distances_int(md, dims, "int16", 32767 - 16)
    f = f0.clone()
    dol.chamfer(f, dims)
    torch.cuda.synchronize()

    def run_ch():
        f.copy_(f0)
        dol.chamfer(f, dims)
    ch = {"workload": "1024^2, 100 points (seed 1), Chamfer 3-4 on int16",
          "gpu_ms": _ev_ms(torch, run_ch, 5) - _ev_ms(torch, lambda: f.copy_(f0), 5)}
    if ref is not None:
        fi = O.init_distances_int(m, dims, np.int16, 32767 - 16, use_ref=True)
        t0 = time.perf_counter()
        O.chamfer(fi, dims, use_ref=True)
        ch["cpu_ref_ms"] = (time.perf_counter() - t0) * 1e3
    res["chamfer_2d_1024"] = ch


def _config2(dol, torch, O, ref, res, L, sp):
    n = 256
    dims = (n, n, n)
    md = torch.empty(dol.mask_words(*dims), dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_shapes_3d(n, n, n, 32, 32, 4, 40, C.c_uint32(7), C.c_void_p(md.data_ptr()), sp))
    occ = float(np.unpackbits(md.cpu().numpy().view(np.uint8)).sum()) / n ** 3
    c2 = {"workload": "256^3, 32 boxes + 32 spheres (4-40, seed 7), signed", "occupancy": occ}
    bor = dol.init_border(md, dims)
    c2["border_init_ms"] = _ev_ms(torch, lambda: dol.init_border(md, dims, out=bor), 3)
    work = bor.clone()
    for meth in ("danielsson", "fastsweep", "jumpflood"):
        def run(meth=meth):
            work.copy_(bor)
            dol.propagate(meth, work, dims, 2)
        run()
        torch.cuda.synchronize()
        c2[f"{meth}_ms"] = _ev_ms(torch, run, 2) - _ev_ms(torch, lambda: work.copy_(bor), 2)
    out = dol.empty_field(dims)
    c2["felzenszwalb_sdf_ms"] = _ev_ms(torch, lambda: dol.edt_mask(md, dims, dol.EDT_SIGNED, out=out), 3)
    # the tool's two-pass -S field: exterior + interior Danielsson (cw = 1), Dist(ext) - Dist(int)
    tp_ws = torch.empty(L.dol_sdf_two_pass_workspace_size(n, n, n, dol.DANIELSSON), dtype=torch.uint8, device="cuda")
    dol.sdf_two_pass(md, dims, "danielsson", want_deltas=False, workspace=tp_ws)
    torch.cuda.synchronize()
    c2["two_pass_danielsson_ms"] = _ev_ms(
        torch, lambda: dol.sdf_two_pass(md, dims, "danielsson", want_deltas=False, workspace=tp_ws), 2)
    del tp_ws
    if ref is not None:
        mh = md.cpu().numpy().view(np.uint32)
        b0 = O.border_init(mh, dims, use_ref=True)
        for meth in ("danielsson", "fastsweep"):
            t0 = time.perf_counter()
            O.propagate(meth, b0, dims, 2, use_ref=True)
            c2[f"cpu_ref_{meth}_ms"] = (time.perf_counter() - t0) * 1e3
        t0 = time.perf_counter()
        O.sdf_two_pass(mh, dims, "danielsson", use_ref=True)
        c2["cpu_ref_two_pass_danielsson_ms"] = (time.perf_counter() - t0) * 1e3
    res["signed_256"] = c2


def _config4(dol, torch, res, L, sp):
    n2, n3 = 4096, 64
    nitems = n2 + n3
    Item = _batch_item_type()
    items = (Item * nitems)()
    tw, tb, tc = C.c_longlong(), C.c_longlong(), C.c_longlong()
    dol.check(L.dol_gen_batch(n2, n3, C.c_uint32(4), items, C.byref(tw), C.byref(tb), C.byref(tc), None, None))
    bm = torch.empty(tw.value, dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_batch(n2, n3, C.c_uint32(4), items, None, None, None, C.c_void_p(bm.data_ptr()), sp))
    bd = torch.empty(tb.value, dtype=torch.uint8, device="cuda")
    bf = torch.empty(tc.value, dtype=torch.float32, device="cuda")
    wsb = L.dol_batch_workspace_size(nitems)
    bws = torch.empty(wsb, dtype=torch.uint8, device="cuda")
    dol.check(L.dol_batch_prepare(nitems, items, C.c_void_p(bws.data_ptr()), C.c_size_t(wsb), sp))
    g = C.c_void_p()
    dol.check(L.dol_batch_graph_create(nitems, C.c_void_p(bm.data_ptr()), C.c_void_p(bd.data_ptr()),
                                       C.c_void_p(bf.data_ptr()), C.c_void_p(bws.data_ptr()), C.byref(g)))
    dol.check(L.dol_graph_launch(g, sp))
    torch.cuda.synchronize()
    t_batch = _ev_ms(torch, lambda: dol.check(L.dol_graph_launch(g, sp)), 3)
    L.dol_graph_destroy(g)
    # per-item loop: one dol_sdf_* call per item on the same buffers, over a sample of items
    sample = list(range(0, nitems, max(1, nitems // 256)))
    ws_loop = torch.empty(64 << 20, dtype=torch.uint8, device="cuda")

    def loop():
        for i in sample:
            it = items[i]
            mptr = C.c_void_p(bm.data_ptr() + 4 * it.mask_word_offset)
            dptr = C.c_void_p(bd.data_ptr() + it.delta_byte_offset)
            fptr = C.c_void_p(bf.data_ptr() + 4 * it.dist_offset)
            if it.d == 1:
                dol.check(L.dol_sdf_2d(it.w, it.h, mptr, dol.DANIELSSON, dptr, fptr, C.c_void_p(ws_loop.data_ptr()),
                                       C.c_size_t(64 << 20), sp))
            else:
                dol.check(L.dol_sdf_3d(it.w, it.h, it.d, mptr, dol.DANIELSSON, dptr, fptr,
                                       C.c_void_p(ws_loop.data_ptr()), C.c_size_t(64 << 20), sp))
    loop()
    torch.cuda.synchronize()
    t_loop = _ev_ms(torch, loop, 1)
    cells = tc.value
    res["batch_4096_64"] = {
        "workload": "4096 polygon masks (side 32-1024, aspect 1-2) + 64 sphere volumes (32-128), signed Danielsson",
        "items": nitems, "cells": cells, "batched_ms": t_batch, "batched_masks_per_s": nitems / t_batch * 1e3,
        "looped_sample_items": len(sample), "looped_ms": t_loop,
        "looped_masks_per_s": len(sample) / t_loop * 1e3,
        "batched_over_looped": (nitems / t_batch) / (len(sample) / t_loop),
        "path": "batched: one persistent launch replayed from a CUDA graph; looped: dol_sdf_* per item"}


def _config5(dol, torch, res):
    """Float sites: forward (seed, plain delta method, |p - site|) against
    forward + loss gradient + backward, 4096 sites (seed 11) on 512^2 and
    128^3, targets from the sites jittered by N(0, 0.5)."""
    out = {}
    for dims in ((512, 512), (128, 128, 128)):
        sites = dol.gen_sites(4096, dims, 11)
        rng = np.random.default_rng(11)
        jit = np.clip(sites + rng.normal(0, 0.5, sites.shape), 0, np.array(dims, np.float32) - 1e-3)
        s = torch.from_numpy(sites).cuda()
        sj = torch.from_numpy(jit.astype(np.float32)).cuda()
        cells = int(np.prod(dims))
        for meth in ("danielsson", "jumpflood"):
            dt, _, _ = dol.sites_forward(sj, dims, meth)

            def fwd(meth=meth):
                return dol.sites_forward(s, dims, meth)

            def fwd_bwd(meth=meth):
                d, own, _ = dol.sites_forward(s, dims, meth)
                return dol.sites_backward(own, s, 2.0 * (d - dt), dims)
            fwd_bwd()
            torch.cuda.synchronize()
            tf = _ev_ms(torch, fwd, 3)
            tfb = _ev_ms(torch, fwd_bwd, 3)
            key = f"{'x'.join(map(str, dims))}_{meth}"
            out[key] = {"fwd_ms": tf, "fwd_bwd_ms": tfb, "fwd_bwd_over_fwd": tfb / tf,
                        "fwd_bwd_gvox_per_s": cells / tfb / 1e6}
    res["sites_4096"] = {"workload": "4096 float sites (seed 11), loss sum (d - d_t)^2, d_t from sites + N(0,0.5)",
                         **out}


def _config3(dol, torch, res, L, sp):
    if True:
        side = 1024
        mdv = torch.empty(dol.mask_words(side, side, side), dtype=torch.int32, device="cuda")
        dol.check(L.dol_gen_value_noise_3d(side, side, side, SPACING, C.c_uint32(SEED), C.c_void_p(mdv.data_ptr()), sp))
        dv = torch.empty((side, side, side, 3), dtype=torch.int16, device="cuda")
        # one untimed run first: its workspace (13.5 GB) comes from the stream-ordered pool
        dol.init_border(mdv, (side,) * 3, out=dv)
        dol.danielsson(dv, (side,) * 3, 2)
        dol.init_border(mdv, (side,) * 3, out=dv)
        torch.cuda.synchronize()
        t = _ev_ms(torch, lambda: dol.danielsson(dv, (side,) * 3, 2), 1)
        res["danielsson_3d_1024"] = {"workload": "1024^3 value noise, signed Danielsson deltas (cw=2)", "gpu_ms": t,
                                     "gvox_per_s": side ** 3 / t / 1e6,
                                     "note": "block schedule: exact fixed-point iteration over blocks of rows "
                                             "(one cooperative launch per z direction), latency-bound"}
        del dv, mdv


def _config_sparse(dol, torch, O, ref, res, L, sp, big=True):
    """The mask EDT where the nearest cell of the other state can be far away:
    the 2D default image (1024^2, 100 points, seed 1) through the mask EDT and
    through the tool's float path (InitDistancesFromBitMask + Felzenszwalb,
    DistanceOcclusionTool.cpp:741-782), and 1024^3 volumes of 2000 points
    (BitMaskAddPoints, seed 1) and of no set voxel, signed."""
    out = {}
    dims = (1024, 1024)
    m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
    md = torch.from_numpy(m.view(np.int32)).cuda()
    f2 = dol.empty_field(dims)
    ws2 = torch.empty(L.dol_edt_mask_2d_workspace_size(*dims), dtype=torch.uint8, device="cuda")
    run = lambda: dol.edt_mask(md, dims, dol.EDT_DIST, out=f2, workspace=ws2)
    run()
    out["edt_2d_1024_points100_ms"] = _ev_ms(torch, run, 5)
    f0 = dol.init_distances(md, dims)
    wf = torch.empty(L.dol_felzenszwalb_2d_workspace_size(*dims), dtype=torch.uint8, device="cuda")
    ff = f0.clone()

    def run_f():
        ff.copy_(f0)
        dol.check(L.dol_felzenszwalb_2d(1024, 1024, C.c_void_p(ff.data_ptr()), C.c_void_p(wf.data_ptr()),
                                        C.c_size_t(wf.numel()), sp))
    run_f()
    out["felzenszwalb_float_2d_1024_points100_ms"] = _ev_ms(torch, run_f, 3) - _ev_ms(torch, lambda: ff.copy_(f0), 3)
    if ref is not None:
        fi = O.init_distances(m, dims, use_ref=True)
        t0 = time.perf_counter()
        O.felzenszwalb(fi, dims, use_ref=True)
        out["cpu_ref_felzenszwalb_2d_1024_points100_ms"] = (time.perf_counter() - t0) * 1e3
    if big:
        side = 1024
        d3 = (side,) * 3
        mh = np.zeros(dol.mask_words(*d3), np.uint32)
        cases = {"points2000": dol.add_points(mh.copy(), d3, 2000, 1), "empty": mh}
        f3 = dol.empty_field(d3)
        ws3 = torch.empty(L.dol_edt_mask_3d_workspace_size(*d3), dtype=torch.uint8, device="cuda")
        for name, mk in cases.items():
            mdv = torch.from_numpy(mk.view(np.int32)).cuda()
            run3 = lambda: dol.edt_mask(mdv, d3, dol.EDT_SIGNED, out=f3, workspace=ws3)
            run3()
            torch.cuda.synchronize()
            L.dol_profile_begin()
            t = _ev_ms(torch, run3, 1)
            names_buf = C.create_string_buffer(4096)
            ms = (C.c_float * 64)()
            n = L.dol_profile_end(names_buf, C.c_size_t(4096), ms, C.c_int(64))
            per = dict(zip(names_buf.value.decode().split("\n")[:n], list(ms)[:n]))
            out[f"edt_3d_1024_{name}_ms"] = t
            out[f"edt_3d_1024_{name}_per_kernel_ms"] = per
        del f3, ws3
    res["edt_sparse"] = out


def _config_occlusion_voxel(dol, torch, O, ref, res):
    """The occlusion sweeps (2D default image; 256^3 value noise, lattice 16,
    seed 3) and the mesh voxeliser (the reference's sample mesh at 256^3), GPU
    against the reference's CPU code (one thread) on the same inputs."""
    import ctypes as C
    out = {}
    for dims in ((1024, 1024), (256, 256, 256)):
        if len(dims) == 2:
            m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
        else:
            m = np.zeros(dol.mask_words(*dims), np.uint32)
            dol.lib().dol_gen_value_noise_3d_host(*dims, SPACING, C.c_uint32(SEED), m.ctypes.data_as(C.c_void_p))
        md = torch.from_numpy(m.view(np.int32)).cuda()
        dw = dol.init_dirw(md, dims)
        run = lambda: dol.occlusion_sweep(dol.init_dirw(md, dims, out=dw), dims)
        run()
        torch.cuda.synchronize()
        key = "x".join(map(str, dims))
        out[f"occlusion_{key}_ms"] = min(_ev_ms(torch, run, 1) for _ in range(3))
        if ref is not None:
            t0 = time.perf_counter()
            O.occlusion_sweep(O.init_dirw(m, dims, use_ref=True), dims, use_ref=True)
            out[f"cpu_ref_occlusion_{key}_ms"] = (time.perf_counter() - t0) * 1e3
    tri = os.path.join(ROOT, "oracle", "_ref", "plant2.tri")
    if os.path.exists(tri):
        idx, v, bb = O.load_tri(tri)
        it, vt = torch.from_numpy(idx).cuda(), torch.from_numpy(v).cuda()
        n = 256
        mv = torch.zeros(dol.mask_words(n, n, n), dtype=torch.int32, device="cuda")
        run = lambda: dol.voxelize(it, vt, bb, (n, n, n), mask=mv)
        run()
        torch.cuda.synchronize()
        out["voxelize_plant2_256_ms"] = min(_ev_ms(torch, run, 1) for _ in range(3))
        out["voxelize_triangles"] = int(idx.shape[0])
        if ref is not None:
            t0 = time.perf_counter()
            O.voxelize(idx, v, bb, (n, n, n), use_ref=True)
            out["cpu_ref_voxelize_plant2_256_ms"] = (time.perf_counter() - t0) * 1e3
    res["occlusion_voxel"] = {"workload": "occlusion sweeps: 1024^2 (100 points, seed 1) and 256^3 value noise; "
                                          "voxeliser: the reference's sample mesh (plant2) at 256^3", **out}


def _batch_item_type():
    class Item(C.Structure):
        _fields_ = [("w", C.c_int), ("h", C.c_int), ("d", C.c_int), ("reserved", C.c_int),
                    ("mask_word_offset", C.c_longlong), ("delta_byte_offset", C.c_longlong),
                    ("dist_offset", C.c_longlong)]
    return Item


# ---------------------------------------------------------------------- our arm ----

def run_dol(args):
    import torch
    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    dol = load_dol()
    L = dol.lib()
    stream = torch.cuda.current_stream()
    sp = C.c_void_p(stream.cuda_stream)
    mw = dol.mask_words(W, H, D)
    mask = torch.empty(mw, dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_value_noise_3d(C.c_int(W), C.c_int(H), C.c_int(D), C.c_int(SPACING), C.c_uint32(SEED),
                                       C.c_void_p(mask.data_ptr()), sp))
    out = torch.empty((D, H, W), dtype=torch.float32, device="cuda")
    wsz = L.dol_edt_mask_3d_workspace_size(W, H, D)
    work = torch.empty(wsz, dtype=torch.uint8, device="cuda")

    def step():
        dol.check(L.dol_edt_mask_3d(C.c_int(W), C.c_int(H), C.c_int(D), C.c_void_p(mask.data_ptr()),
                                    C.c_void_p(out.data_ptr()), C.c_int(dol.EDT_SIGNED),
                                    C.c_void_p(work.data_ptr()), C.c_size_t(wsz), sp))

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    # per-kernel times for the roofline, on the launching stream (a separate, untimed pass)
    L.dol_profile_begin()
    for _ in range(max(1, min(args.steps, 3))):
        step()
    names_buf = C.create_string_buffer(4096)
    ms = (C.c_float * 64)()
    n = L.dol_profile_end(names_buf, C.c_size_t(4096), ms, C.c_int(64))
    names = names_buf.value.decode().split("\n")[:n]
    per = {}
    for nm, t in zip(names, list(ms)[:n]):
        per.setdefault(nm, []).append(t)
    kern = {k: float(np.mean(v)) for k, v in per.items()}
    launches_per_step = len(kern)   # kernels of one step: one per profiled scope

    clocks = ClockSampler(local)
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_total = e0.elapsed_time(e1)
    if pg:
        pg.barrier()
    clk = clocks.stop()
    ms_total = max_over_ranks(ms_total, pg)
    ms_step = ms_total / args.steps
    value = job_gvox_per_s(ws, W * H * D, ms_step * 1e-3)

    # e2e: host mask in (pinned), host field out (pinned), through the host-buffer C ABI call
    e2e = None
    if not args.no_e2e:
        hmask = torch.empty(mw, dtype=torch.int32, pin_memory=True)
        hmask.copy_(mask.cpu())
        hout = torch.empty((D, H, W), dtype=torch.float32, pin_memory=True)
        ts = []
        for i in range(args.e2e_warmup + args.e2e_steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            dol.check(L.dol_edt_mask_3d_host(C.c_int(W), C.c_int(H), C.c_int(D), C.c_void_p(hmask.data_ptr()),
                                             C.c_void_p(hout.data_ptr()), C.c_int(dol.EDT_SIGNED)))
            if i >= args.e2e_warmup:
                ts.append(time.perf_counter() - t)
        e2e_s = max_over_ranks(float(np.mean(ts)), pg)
        e2e = {"value": job_gvox_per_s(ws, W * H * D, e2e_s), "unit": "Gvoxels/s", "h2d_bytes_per_step": mw * 4,
               "d2h_bytes_per_step": W * H * D * 4, "ms_per_step": e2e_s * 1e3,
               "path": "dol_edt_mask_3d_host, pinned host buffers"}

    if pg:
        pg.barrier()
    if rank != 0:
        if pg:
            pg.destroy_process_group()
        return

    peak, peak_kind = measured_peak()
    dom = max(kern, key=kern.get) if kern else None
    roof = None
    if dom:
        alg = PASS_BYTES.get(dom, 0.0) * W * H * D
        ach = alg / (kern[dom] * 1e-3) / 1e9
        traffic = None
        tf = os.path.join(ROOT, "profiles", "edt_traffic.json")
        if os.path.exists(tf):
            try:
                traffic = json.load(open(tf)).get(dom)
            except Exception:
                traffic = None
        roof = {"bound": "hbm", "kernel": dom, "achieved": ach, "peak": peak, "peak_kind": peak_kind,
                "unit": "GB/s", "frac": ach / peak, "traffic": traffic,
                "algorithmic_bytes_per_launch": alg, "launch_ms": kern[dom],
                "per_kernel_ms": kern,
                "per_kernel_frac": {k: PASS_BYTES.get(k, 0) * W * H * D / (v * 1e-3) / 1e9 / peak
                                    for k, v in kern.items()}}
    cpu = None
    if ws == 1 and not args.no_cpu:
        cpu = cpu_reference_sample(steps=args.cpu_steps)
    configs = None
    if not args.no_configs:
        del work
        torch.cuda.empty_cache()
        configs = measure_configs(dol, torch, cpu=(ws == 1 and not args.no_cpu), big=not args.no_big)
    line = {
        "metric": METRIC, "value": value, "unit": "Gvoxels/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (exact integer EDT) -> f32", "data": "synthetic",
        "config": bench_config(ws),
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": launches_per_step * args.steps,
        "configs": configs,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def danielsson_only(shape):
    """Signed Danielsson (border init, cw = 2) on a value-noise volume of the
    given shape, run twice with CUDA events around each run."""
    import torch
    dol = load_dol()
    L = dol.lib()
    w, h, d = (int(v) for v in shape.split("x"))
    dims = (w, h, d)
    md = torch.empty(dol.mask_words(*dims), dtype=torch.int32, device="cuda")
    dol.check(L.dol_gen_value_noise_3d(w, h, d, SPACING, C.c_uint32(SEED), C.c_void_p(md.data_ptr()), None))
    base = dol.init_border(md, dims)
    work = base.clone()
    times = []
    for _ in range(2):
        work.copy_(base)
        torch.cuda.synchronize()
        times.append(_ev_ms(torch, lambda: dol.danielsson(work, dims, 2), 1))
    dol.sync()
    print(json.dumps({"danielsson_signed": shape, "ms": times}), flush=True)


# ------------------------------------------------------------ single kernels ----
# One small workload per kernel family, run `reps` times after one untimed run,
# each timed with CUDA events: the commands the ncu summaries under profiles/
# are made with (inputs larger than L2 where the family allows, a few GB at
# most on the device).

def _case_inputs(dol, torch, L, kind, n):
    dims = (n, n, n)
    md = torch.empty(dol.mask_words(*dims), dtype=torch.int32, device="cuda")
    if kind == "noise":
        dol.check(L.dol_gen_value_noise_3d(n, n, n, SPACING, C.c_uint32(SEED), C.c_void_p(md.data_ptr()), None))
    elif kind == "shapes":
        dol.check(L.dol_gen_shapes_3d(n, n, n, 32 * n // 256, 32 * n // 256, 4 * n // 256, 40 * n // 256,
                                      C.c_uint32(7), C.c_void_p(md.data_ptr()), None))
    else:   # 2000 points per 1024^3, scaled
        mh = np.zeros(dol.mask_words(*dims), np.uint32)
        md = torch.from_numpy(dol.add_points(mh, dims, max(1, 2000 * n ** 3 // 1024 ** 3), 1).view(np.int32)).cuda()
    return dims, md


def run_case(name, reps=2):
    import torch
    dol = load_dol()
    L = dol.lib()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    fn, note = None, ""
    if name.startswith("edt_"):                    # edt_noise_512, edt_points_512, edt_shapes_256
        _, kind, n = name.split("_")
        dims, md = _case_inputs(dol, torch, L, kind, int(n))
        out = dol.empty_field(dims)
        ws = torch.empty(L.dol_edt_mask_3d_workspace_size(*dims), dtype=torch.uint8, device="cuda")
        fn = lambda: dol.edt_mask(md, dims, dol.EDT_SIGNED, out=out, workspace=ws)
    elif name in ("border_256", "danielsson_256", "fastsweep_256", "jumpflood_256", "dist_256"):
        dims, md = _case_inputs(dol, torch, L, "shapes", 256)
        bor = dol.init_border(md, dims)
        work = bor.clone()
        f = dol.empty_field(dims)
        meth = name.split("_")[0]
        if meth == "border":
            fn = lambda: dol.init_border(md, dims, out=work)
        elif meth == "dist":
            dol.danielsson(work, dims, 2)
            fn = lambda: dol.check(L.dol_deltas_to_dist_3d(*dims, C.c_void_p(work.data_ptr()), 2,
                                                            C.c_void_p(md.data_ptr()), C.c_void_p(f.data_ptr()), None))
        else:
            def fn(meth=meth):
                work.copy_(bor)
                dol.propagate(meth, work, dims, 2)
    elif name == "chamfer_1024":
        dims = (1024, 1024)
        m = dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
        md = torch.from_numpy(m.view(np.int32)).cuda()
        f0 = dol.init_distances_int(md, dims, "int16", 32767 - 16)
        f = f0.clone()

        def fn():
            f.copy_(f0)
            dol.chamfer(f, dims)
    elif name.startswith("occlusion_"):           # occlusion_1024 (2D), occlusion_128 / _256, occlusion_io_256
        n = int(name.split("_")[-1])
        if n == 1024:
            dims = (1024, 1024)
            md = torch.from_numpy(dol.add_points(np.zeros(dol.mask_words(*dims), np.uint32), dims, 100, 1)
                                  .view(np.int32)).cuda()
        else:
            dims, md = _case_inputs(dol, torch, L, "noise", n)
        dw = dol.init_dirw(md, dims)
        if "_io_" in name:
            dout = dw.clone()
            fn = lambda: dol.occlusion_sweep_io(dw, dout, dims)
        else:
            fn = lambda: dol.occlusion_sweep(dol.init_dirw(md, dims, out=dw), dims)
    elif name.startswith("voxel_"):                # voxel_256: the reference's sample mesh
        import oracle as O
        n = int(name.split("_")[1])
        idx, v, bb = O.load_tri(os.path.join(ROOT, "oracle", "_ref", "plant2.tri"))
        it, vt = torch.from_numpy(idx).cuda(), torch.from_numpy(v).cuda()
        m = torch.zeros(dol.mask_words(n, n, n), dtype=torch.int32, device="cuda")
        fn = lambda: dol.voxelize(it, vt, bb, (n, n, n), mask=m)
    elif name == "batch":
        res = {}
        _config4(dol, torch, res, L, C.c_void_p(torch.cuda.current_stream().cuda_stream))
        print(json.dumps({"case": name, **res["batch_4096_64"]}), flush=True)
        return
    elif name.startswith("sites_"):                # sites_512: 4096 sites, Danielsson forward + backward
        dims = (512, 512)
        s = torch.from_numpy(dol.gen_sites(4096, dims, 11)).cuda()

        def fn():
            d, own, _ = dol.sites_forward(s, dims, "danielsson")
            dol.sites_backward(own, s, 2.0 * d, dims)
    else:
        raise SystemExit(f"unknown case {name}")
    fn()
    torch.cuda.synchronize()
    ms = [_ev_ms(torch, fn, 1) for _ in range(reps)]
    dol.sync()
    print(json.dumps({"case": name, "ms": ms, "note": note}), flush=True)


CASES = ["edt_noise_512", "edt_points_512", "edt_shapes_256", "border_256", "danielsson_256", "fastsweep_256",
         "jumpflood_256", "dist_256", "chamfer_1024", "occlusion_1024", "occlusion_128", "occlusion_256",
         "occlusion_io_256", "voxel_256", "batch",
         "sites_512"]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dol", choices=["dol", "reference"])
    ap.add_argument("--cpu-steps", type=int, default=3, help="timed steps of the CPU baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--side", type=int, default=SIDE, help="volume side (1024 = the benchmarked workload)")
    ap.add_argument("--no-configs", action="store_true", help="skip the per-configuration measurements")
    ap.add_argument("--no-big", action="store_true", help="skip Danielsson on the 1024^3 volume")
    ap.add_argument("--only", default=None,
                    help="comma list of c1..c8: run only these per-configuration measurements (no headline)")
    ap.add_argument("--case", default=None, choices=CASES, help="run one kernel family's small workload (profiling)")
    ap.add_argument("--danielsson", default=None, metavar="WxHxD",
                    help="only time signed Danielsson on a WxHxD value-noise volume (twice; for profiling)")
    args = ap.parse_args()
    global W, H, D
    W = H = D = args.side
    if args.impl == "reference":
        run_reference(args)
    elif args.case:
        run_case(args.case)
    elif args.danielsson:
        danielsson_only(args.danielsson)
    elif args.only:
        import torch
        dol = load_dol()
        print(json.dumps(measure_configs(dol, torch, cpu=not args.no_cpu, big=True,
                                         only=set(args.only.split(",")))), flush=True)
    else:
        run_dol(args)


if __name__ == "__main__":
    main()
