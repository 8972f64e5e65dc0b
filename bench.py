#!/usr/bin/env python3
"""Benchmark of the photon-transport hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch: ``--photons`` photons of the
workload traced through the mesh, tallies zeroed before and complete after.
Photons are sharded by index range across ranks (weak scaling: every rank traces
the same number of photons per step); the integer tallies are summed over ranks
with one NCCL all-reduce per step, inside the timed region.

value  photons/s of the whole job from CUDA-event device time (inputs resident),
       max over ranks; an L2-sized buffer is rewritten between timed steps.
e2e    the same metric through the public API with host buffers: every step sets
       the mesh (BVH build + upload), media, source and grid from host arrays,
       runs, and copies all tallies back to the host.
roofline  FP32 issue bound: algorithmic FLOPs per photon
       F = 64*E_s + 48*E_b + 40*E_q (scatter events, boundary events, queries per
       photon, counted by the kernel) over the measured FP32 FMA peak of the device.
cpu_baseline / --impl reference  the reference kernel source compiled for the CPU
       (oracle/_ref/libclref.so) on all host cores, plus the launcher's host binning,
       on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "photons/s on 1 B200: plain vs batched at <=1% rel. error; gradient cost/forward"
L2_BYTES = 126 * 1024 * 1024


def env_int(k, d):
    try:
        return int(os.environ.get(k, d))
    except ValueError:
        return d


def load_workload(name, photons):
    from lightpropagation_b200 import workloads
    w = workloads.WORKLOADS[name]()
    if photons:
        w.n_photons = int(photons)
    return w


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.gpu), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------ reference arm
def reference_lib():
    path = os.path.join(ROOT, "oracle", "_ref", "libclref.so")
    if not os.path.isfile(path):
        return None, "oracle/_ref/libclref.so not built (the reference checkout was absent at build time)"
    L = C.CDLL(path)
    fp, ip = C.POINTER(C.c_float), C.POINTER(C.c_int32)
    L.clref_run_mt.argtypes = [C.c_int, C.c_float, fp, ip, fp, C.c_float, C.c_float, C.c_int, fp, fp, C.c_long,
                               C.c_long, fp, fp, fp, fp, fp, ip, fp, fp, ip, C.c_long, C.c_int]
    L.clref_run_mt.restype = C.c_int
    L.clref_psnr_state.argtypes = [C.c_int, fp, ip]
    return L, None


def _ptr(a, t=C.c_float):
    return a.ctypes.data_as(C.POINTER(t))


def run_reference_sample(w, n, threads, seed=1):
    """Trace n photons with the reference kernel on `threads` host threads; bin the
    exit records like ExecKernel.  Returns (seconds, photons)."""
    L, why = reference_lib()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    case = po.Case(tri=w.tri, nrm=w.nrm, med=w.med, nmuasg=w.nmuasg, p_start=w.p_start, v_start=w.v_start,
                   ep0xyz=w.ep0xyz, dimensions=w.dimensions, det_grid=w.det_grid, fetal_id=w.fetal_id,
                   chance=w.chance, w_threshold=w.w_threshold, factor=w.factor)
    g = po.geometry(case)
    T = w.tri.shape[0]
    tri = np.zeros((T + 1) * 9, np.float32); tri[9:] = w.tri.ravel()
    nrm = np.zeros((T + 1) * 3, np.float32); nrm[3:] = w.nrm.ravel()
    med = np.zeros((T + 1) * 2, np.int32); med[2:] = w.med.ravel()
    cells = g.rz_nr * g.rz_nz
    pad = 4 * cells + 100000
    stride = cells + 2 * pad
    rz = np.zeros((threads * stride, 3), np.float32)
    st = np.zeros(56, np.float32)
    ix = np.zeros(3, np.int32)
    L.clref_psnr_state(seed, _ptr(st), _ptr(ix, C.c_int32))
    rec = np.zeros((n, 8), np.float32)
    dims = np.array([g.dimx, g.dimy, g.dimz], np.float32)
    occ = np.array([n], np.int32)
    nm = np.ascontiguousarray(w.nmuasg, np.float32).ravel()
    t0 = time.perf_counter()
    L.clref_run_mt(T, w.factor, _ptr(np.ascontiguousarray(w.v_start, np.float32)), _ptr(occ, C.c_int32),
                   _ptr(np.ascontiguousarray(w.p_start, np.float32)), w.chance, w.w_threshold, w.fetal_id,
                   _ptr(rec), _ptr(rz), stride, pad, _ptr(dims), _ptr(np.ascontiguousarray(w.ep0xyz, np.float32)),
                   _ptr(np.ascontiguousarray(w.det_grid, np.float32)),
                   C.cast(C.c_void_p(tri.ctypes.data + 36), C.POINTER(C.c_float)),
                   C.cast(C.c_void_p(nrm.ctypes.data + 12), C.POINTER(C.c_float)),
                   C.cast(C.c_void_p(med.ctypes.data + 8), C.POINTER(C.c_int32)), _ptr(nm), _ptr(st),
                   _ptr(ix, C.c_int32), n, threads)
    bin_exit_records(rec, g, w.det_grid)
    return time.perf_counter() - t0, n


def bin_exit_records(rec, g, dg):
    """ExecKernel's host binning (CalculatePropagation.cpp:1553-1626), vectorised."""
    hx, hy = g.dimx // 2, g.dimy // 2
    sft = np.zeros((g.sft_ny, g.sft_nx, 3), np.float64)
    rtd = np.zeros((g.dimAlpha, g.dimR, 3), np.float64)
    with np.errstate(invalid="ignore"):
        x = np.clip(np.nan_to_num(rec[:, 0] / dg[0]).astype(np.int64), -hx, hx)
        y = np.clip(np.nan_to_num(rec[:, 1] / dg[1]).astype(np.int64), -hy, hy)
        a = np.nan_to_num((rec[:, 6] * np.float32(180)).astype(np.float64) / np.pi / float(dg[5]))
        r = np.nan_to_num(rec[:, 7] / dg[3])
    a = np.clip(a, -1e9, 1e9).astype(np.int64).clip(0, g.dimAlpha - 1)
    r = np.clip(r, -1e9, 1e9).astype(np.int64).clip(0, g.dimR - 1)
    for c in range(3):
        np.add.at(sft[:, :, c], (y + hy, x + hx), rec[:, 3 + c])
        np.add.at(rtd[:, :, c], (a, r), rec[:, 3 + c])
    return sft, rtd


def reference_arm(args, w):
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    L, why = reference_lib()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    # calibrate a bounded sample (a few seconds per step)
    dt, n0 = run_reference_sample(w, threads, threads)
    per_photon = dt / n0
    n = int(max(threads, min(w.n_photons, 3.0 / max(per_photon, 1e-9))))
    for _ in range(args.warmup):
        run_reference_sample(w, max(threads, n // 4), threads)
    tot_t, tot_n = 0.0, 0
    for _ in range(args.steps):
        t, k = run_reference_sample(w, n, threads)
        tot_t += t
        tot_n += k
    v = tot_n / tot_t
    line = {"metric": METRIC, "value": v, "unit": "photons/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": w.name, "photons_per_step": n, "triangles": int(w.n_tri),
                       "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": v, "unit": "photons/s", "cores": threads, "kind": "reference",
                             "sample": f"{n} photons per step of {w.name} (reference kernel source compiled for "
                                       f"the CPU + host binning)"},
            "e2e": {"value": v, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ our arm
def fp32_flops_per_photon(c, n):
    """Algorithmic FP32 work per photon.  E_q counts the queries of the reference's
    algorithm (one per loop iteration, FindTriangleInPath at .cl:1379), not the ones the
    kernel executes after safety-grid skips."""
    es, eb = c["scatter"] / n, c["boundary"] / n
    eq = es + eb
    return 64 * es + 48 * eb + 40 * eq, es, eb, eq


def traffic_per_photon(workload):
    """DRAM bytes per photon of the transport kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", f"transport_kernel_{workload}.md")
    if not os.path.isfile(path):
        return None
    import re
    m = re.search(r"dram_bytes_per_photon:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def ours_arm(args, w):
    import torch
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from lightpropagation_b200 import Simulation
    from lightpropagation_b200.propagation import fp32_peak_tflops
    n = w.n_photons
    sim = Simulation(local)
    w.apply(sim, seed=0x4C50)
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")

    red = []
    if dist is not None:
        sim.run(0)
        d = sim.device_tallies()

        class _CA:
            def __init__(self, ptr, cnt):
                self.__cuda_array_interface__ = {"shape": (cnt,), "typestr": "<i8", "data": (ptr, False),
                                                 "version": 3}
        for name in ("sft", "rtd", "rz", "vox", "rbins", "region", "det", "counters"):
            cnt = getattr(d, "n_" + name)
            if cnt > 0:
                red.append(torch.as_tensor(_CA(getattr(d, name), cnt), device=f"cuda:{local}"))

    def step(i):
        sim.zero()
        first = (i * world + rank) * n
        sim.run(n, first)
        ms = sim.kernel_ms()
        if dist is not None:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            for t in red:
                dist.all_reduce(t)
            ev1.record()
            ev1.synchronize()
            ms += ev0.elapsed_time(ev1)
        return ms

    for i in range(args.warmup):
        step(i)
    peak = fp32_peak_tflops(local)
    clocks = ClockSampler(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    dev_ms = 0.0
    counters = None
    for i in range(args.steps):
        flush.fill_(float(i))           # rewrite a 2x-L2 buffer between timed steps
        torch.cuda.synchronize()
        dev_ms += step(args.warmup + i)
        if i == args.steps - 1:
            counters = sim.tallies()["counters"]
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    wall = time.perf_counter() - wall0
    clk = clocks.stop()
    st = sim.stats()
    t_max = dev_ms
    if dist is not None:
        t = torch.tensor([dev_ms], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    total_photons = n * world * args.steps
    value = total_photons / (t_max * 1e-3)

    # e2e through the public API with host buffers (fresh context state every step)
    e2e_v = h2d = d2h = None
    if rank == 0 or world > 1:
        e2e_t = 0.0
        for i in range(max(1, min(args.steps, 3))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            with Simulation(local) as s2:
                w.apply(s2, seed=0x4C50 + i)
                s2.run(n, rank * n)
                s2.tallies()
                st2 = s2.stats()
            e2e_t += time.perf_counter() - t0
            h2d, d2h = st2["h2d_bytes"], st2["d2h_bytes"]
        e2e_v = n * world * max(1, min(args.steps, 3)) / e2e_t

    if dist is not None:
        red.clear()
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        sim.close()
        return 0

    # roofline of the transport kernel (counters are global after the all-reduce)
    per_launch_photons = n * world
    F, es, eb, eq = fp32_flops_per_photon(counters, per_launch_photons)
    avg_kernel_ms = st["last_kernel_ms"]
    achieved = F * n / (avg_kernel_ms * 1e-3) / 1e12
    tpp = traffic_per_photon(w.name)
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None,
            "traffic": (tpp * n) if tpp is not None else None,
            "peak_source": "FP32 FMA peak measured in-run by lp_fp32_peak (MEASURED_PEAKS.json has no FP32 figure)",
            "flops_per_photon": F,
            "events_per_photon": {"scatter": es, "boundary": eb, "query": eq,
                                  "query_executed": counters["query"] / per_launch_photons,
                                  "query_skipped_by_safety_grid": counters["safe_skip"] / per_launch_photons}}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            dt, n0 = run_reference_sample(w, threads, threads)
            m = int(max(threads, min(w.n_photons, 12.0 / max(dt / n0, 1e-9))))
            dt, k = run_reference_sample(w, m, threads)
            cpu = {"value": k / dt, "unit": "photons/s", "cores": threads, "kind": "reference",
                   "sample": f"{k} photons of {w.name}: reference kernel source compiled for the CPU "
                             f"(oracle/_ref) on {threads} threads + host binning"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "photons/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    line = {"metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": w.name, "photons_per_step_per_gpu": n, "triangles": int(w.n_tri),
                       "parallelism": f"photon ranges x{world}" + (" + NCCL all-reduce of tallies" if world > 1 else ""),
                       "l2": "2x L2 buffer rewritten between timed steps",
                       "grid": st["grid"], "block": st["block"], "bvh_nodes": st["n_nodes"],
                       "bvh_nodes_in_smem": st["nodes_smem"], "tris_in_smem": st["tris_smem"]},
            "wall_s": wall, "clocks": clk, "gpu_launches": args.steps,
            "e2e": {"value": e2e_v, "unit": "photons/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "roofline": roof, "cpu_baseline": cpu}
    print(json.dumps(line))
    sim.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="plain_slab")
    ap.add_argument("--photons", type=int, default=0, help="photons per step per GPU (default: workload's)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    w = load_workload(args.workload, args.photons)
    if args.impl == "reference":
        return reference_arm(args, w)
    return ours_arm(args, w)


if __name__ == "__main__":
    sys.exit(main())
