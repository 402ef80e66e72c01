"""Benchmark: signed distance field of a 1024^3 volume on one B200 per rank.

Workload (the large 3D SDF throughput case): a 1024^3 1-bit volume of 3D value
noise (lattice spacing 16, uniform lattice values from the reference's LCG,
seed 3, trilinear, thresholded at 1/2, ~50% occupied).  One step = the
mask-driven exact Felzenszwalb transform producing the signed float field
(distance to set voxels minus distance to clear voxels) from a device-resident
mask.  Metric: Gvoxels/s of the whole job.  Inputs and outputs (128 MiB mask,
4 GiB field) are far larger than L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl dol|reference]

--impl reference times the reference's own CPU code for the same output on a
bounded sub-volume (the reference's 1D Felzenszwalb routine applied along z,
y, x -- it has no 3D driver -- twice, for the two signs, on all host cores).
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
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
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
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


# ---------------------------------------------------------------- reference arm ----

def cpu_reference_sample(side=256, reps=None, target_s=10.0, threads=None):
    """The reference's CPU code on a side^3 corner of the same noise volume:
    signed field from two transforms (distance to set, distance to clear) with
    the reference's 1D Felzenszwalb routine along z, y, x.  Returns Gvox/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    dol = load_dol()
    threads = threads or os.cpu_count() or 1
    kind = "reference" if O.ref() is not None else "port"
    n = side
    # a side^3 volume of the same noise (same spacing, seed and threshold)
    words = np.zeros(((n + 31) // 32) * n * n, np.uint32)
    dol.lib().dol_gen_value_noise_3d_host(C.c_int(n), C.c_int(n), C.c_int(n), C.c_int(SPACING), C.c_uint32(SEED),
                                          words.ctypes.data_as(C.c_void_p))
    b = O.mask_to_bool(words, (n, n, n))
    big = np.float32(np.finfo(np.float32).max)
    done, t0, reps_done = False, time.perf_counter(), 0
    elapsed = 0.0
    while not done:
        t1 = time.perf_counter()
        f_occ = np.where(b, np.float32(0), big).astype(np.float32)
        f_emp = np.where(b, big, np.float32(0)).astype(np.float32)
        if kind == "reference":
            e_occ = O.felzenszwalb(f_occ, (n, n, n), use_ref=True, threads=threads)
            e_emp = O.felzenszwalb(f_emp, (n, n, n), use_ref=True, threads=threads)
        else:
            e_occ = O.felzenszwalb(f_occ, (n, n, n))
            e_emp = O.felzenszwalb(f_emp, (n, n, n))
        _ = np.sqrt(e_occ) - np.sqrt(e_emp)
        elapsed += time.perf_counter() - t1
        reps_done += 1
        done = (reps is not None and reps_done >= reps) or (reps is None and time.perf_counter() - t0 >= target_s)
    vox = reps_done * n ** 3
    return {"value": vox / elapsed / 1e9, "unit": "Gvoxels/s", "cores": threads if kind == "reference" else 1,
            "kind": kind,
            "sample": f"{n}^3 volume of the same noise x{reps_done}: two 3D transforms with the reference's "
                      f"1D Felzenszwalb (DistanceOcclusionLib.cpp:1026-1062) along z,y,x + sqrt/sub"}


def run_reference(args):
    ws, rank, local = dist_setup()
    if rank != 0:
        return
    t_per = []
    res = None
    for i in range(args.warmup + args.steps):
        t = time.perf_counter()
        res = cpu_reference_sample(side=args.cpu_side, reps=1)
        if i >= args.warmup:
            t_per.append(time.perf_counter() - t)
    vox = args.cpu_side ** 3
    value = vox / float(np.mean(t_per)) / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gvoxels/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(t_per)) * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample": f"{args.cpu_side}^3 volume of the same noise per step (CPU)"},
        "cpu_baseline": {"value": value, "unit": "Gvoxels/s", "cores": res["cores"], "kind": res["kind"],
                         "sample": res["sample"]},
        "e2e": {"value": value, "unit": "Gvoxels/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


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
    if pg:
        t = torch.tensor([ms_total], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms_total = float(t.item())
    ms_step = ms_total / args.steps
    value = ws * W * H * D / (ms_step * 1e-3) / 1e9

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
        e2e_s = float(np.mean(ts))
        if pg:
            t = torch.tensor([e2e_s], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            e2e_s = float(t.item())
        e2e = {"value": ws * W * H * D / e2e_s / 1e9, "unit": "Gvoxels/s", "h2d_bytes_per_step": mw * 4,
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
        cpu = cpu_reference_sample(side=args.cpu_side, target_s=args.cpu_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": "Gvoxels/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (exact integer EDT) -> f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "voxels_per_gpu": W * H * D, "parallelism": f"replicas x{ws}",
                   "l2": "inputs and outputs > L2 (128 MiB mask in, 4 GiB field out); no flush needed"},
        "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk,
        "gpu_launches": 3 * args.steps,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dol", choices=["dol", "reference"])
    ap.add_argument("--cpu-side", type=int, default=256)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-warmup", type=int, default=1)
    ap.add_argument("--side", type=int, default=SIDE, help="volume side (1024 = the benchmarked workload)")
    args = ap.parse_args()
    global W, H, D
    W = H = D = args.side
    if args.impl == "reference":
        run_reference(args)
    else:
        run_dol(args)


if __name__ == "__main__":
    main()
