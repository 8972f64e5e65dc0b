#!/usr/bin/env python3
"""Benchmark of the photon-transport hot path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload NAME]

A step is one pass of the hot path over one batch: ``--photons`` photons (1e8 by
default for the abdomen, the workload's stated count per launch) traced through the
mesh in one launch, tallies zeroed before and complete after.  The default workload is
the curved-mesh abdomen (202,500 triangles, fibre source, six ring detectors) at 660 nm
and at 940 nm: steps alternate between the two optical-property tables on one mesh, so
a job of K steps traces about K/2 batches at each wavelength.  ``--photons 10000000``
runs the shorter 1e7-photon launches.  ``--workload plain_slab`` is the small 3-layer
slab.  Photons are sharded by index range across ranks (weak
scaling: every rank traces the same number of photons per step); the integer
tallies are summed over ranks with one NCCL all-reduce per launch, inside the
timed region.

detector_error  relative standard error of every ring detector's signal after one
       launch, and the photon count that brings the farthest ring to 1%.

value  photons/s of the whole job from CUDA-event device time (inputs resident),
       max over ranks; an L2-sized buffer is rewritten between timed steps.
e2e    the same metric through the public API with host buffers: every step sets
       the mesh (BVH build + upload), media, source and grid from host arrays,
       runs, and copies all tallies back to the host.
roofline  FP32 issue bound: algorithmic FLOPs per photon
       F = 64*E_s + 48*E_b + 40*E_q (scatter events, boundary events, queries per
       photon, counted by the kernel) over the measured FP32 FMA peak of the device;
       beside it the L2-atomic fraction: absorption and exit deposits per second over
       the measured rate of 64-bit atomic adds to an L2-resident buffer.
config1_slab  the like-for-like comparison: the 3-layer slab (32 triangles, pencil beam,
       reference behaviours on, 1e6 photons) on the GPU and through the reference's
       own kernel source on the host cores, the same physics on both sides.
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


def load_cases(name, photons):
    """The workloads the steps trace, in turn.  ``curved_abdomen`` (the default) is the
    curved-mesh abdomen at 660 nm and at 940 nm: one mesh, two optical-property tables,
    1e8 photons per launch."""
    import dataclasses
    from lightpropagation_b200 import workloads
    if name == "curved_abdomen":
        w = workloads.curved_abdomen(wavelength=660, n_photons=100_000_000)
        nm940 = np.array(workloads.ABDOMEN_MEDIA[940], np.float32)
        cases = [w, dataclasses.replace(w, nmuasg=nm940, name=w.name.replace("660nm", "940nm"))]
    else:
        cases = [workloads.WORKLOADS[name]()]
    for c in cases:
        if photons:
            c.n_photons = int(photons)
    return cases


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def ring_rse(det, n):
    """Relative standard error of each ring detector's mean signal per photon, from the
    fixed-point sums (sum w, sum w^2) over n photons."""
    s = det[:, 0].astype(np.float64) / 2.0 ** 32
    s2 = det[:, 1].astype(np.float64) / 2.0 ** 32
    var = np.maximum(s2 - s * s / n, 0.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        return np.where(s > 0, np.sqrt(var) / s, np.inf)


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


def reference_sample_size(cases, threads, seconds):
    """Photons per case for a reference sample of about `seconds` of host time."""
    dt = sum(run_reference_sample(c, threads, threads)[0] for c in cases)
    per_photon = dt / (threads * len(cases))
    return int(max(threads, min(cases[0].n_photons, seconds / len(cases) / max(per_photon, 1e-9))))


def reference_sample(cases, n, threads):
    """n photons of every case through the reference kernel: (seconds, photons)."""
    tot_t, tot_n = 0.0, 0
    for c in cases:
        t, k = run_reference_sample(c, n, threads)
        tot_t += t
        tot_n += k
    return tot_t, tot_n


def workload_label(args, cases):
    if len(cases) == 1:
        return cases[0].name
    return f"{args.workload}: " + " + ".join(c.name for c in cases)


def reference_arm(args, cases):
    """The reference's own CPU implementation of the path on all host cores: each step a
    bounded sample of the step's case (cases alternate as in our arm), plus the
    like-for-like config-1 slab figure."""
    rank = env_int("RANK", 0)
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    L, why = reference_lib()
    if L is None:
        print(json.dumps({"impl": "reference", "unavailable": why}))
        return 0
    n = reference_sample_size(cases, threads, 3.0 * len(cases))   # a bounded sample, a few seconds per step
    for i in range(args.warmup):
        reference_sample([cases[i % len(cases)]], max(threads, n // 8), threads)
    tot_t, tot_n = 0.0, 0
    for i in range(args.steps):
        t, k = reference_sample([cases[i % len(cases)]], n, threads)
        tot_t += t
        tot_n += k
    v = tot_n / tot_t
    label = workload_label(args, cases)
    slab = None
    if args.workload == "curved_abdomen" and not args.no_slab:
        from lightpropagation_b200 import workloads
        ws = workloads.plain_slab()
        m = reference_sample_size([ws], threads, 10.0)
        dt, k = reference_sample([ws], m, threads)
        slab = {"workload": ws.name, "reference_photons_per_s": k / dt,
                "reference_sample": f"{k} photons on {threads} threads",
                "same_physics": "pencil beam, reference behaviours Q3/Q4/Q10 on, on both sides"}
    line = {"metric": METRIC, "value": v, "unit": "photons/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": {"workload": label, "photons_per_step_per_gpu": n, "photons_per_launch": n,
                       "triangles": int(cases[0].n_tri), "steps_alternate": [c.name for c in cases],
                       "parallelism": f"{threads} host threads"},
            "cpu_baseline": {"value": v, "unit": "photons/s", "cores": threads, "cpu_model": cpu_model(),
                             "kind": "reference",
                             "sample": f"{n} photons per step of {label}: the reference kernel source compiled for "
                                       f"the CPU (oracle/_ref; a pencil beam, its only source; brute-force "
                                       f"triangle search) + ExecKernel's host binning"},
            "e2e": {"value": v, "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "config1_slab": slab}
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


def traffic_of(workload):
    """DRAM bytes of one transport launch and that launch's photon count, from the
    committed ncu summary (dram__bytes_read.sum + dram__bytes_write.sum)."""
    path = os.path.join(ROOT, "profiles", f"transport_kernel_{workload}.md")
    if not os.path.isfile(path):
        return None, None
    import re
    text = open(path).read()
    b = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", text)
    p = re.search(r"dram_bytes_launch_photons:\s*([0-9.eE+]+)", text)
    return (float(b.group(1)) if b else None), (int(float(p.group(1))) if p else None)


def batched_section(args, local):
    """Plain vs batched forms on the batched abdomen workload: the curved-abdomen mesh plus
    8 variants (fetal-head depth, fat thickness), `--batch-instances` optical-property
    instances at 660/940 nm with log-uniform budgets in [--batch-min, --batch-max].
    plain  = one lp_run per instance on its mesh's context (device time of the launches);
    batched = one lp_batch_run (graph: zero all tallies, a persistent launch of its own
    for every instance of at least 2^20 photons, one persistent batch launch for the rest).
    Both trace the same photons and give bit-identical tallies, so the detector errors are
    matched by construction."""
    from lightpropagation_b200 import Batch, Instance, Simulation, workloads
    spec = workloads.batched_abdomen(n_instances=args.batch_instances, budget=(args.batch_min, args.batch_max))
    sims = [m.apply(Simulation(local), seed=0x4C50) for m in spec.meshes]
    insts = [Instance(context=x["mesh"], nmuasg=x["nmuasg"], n_photons=x["n_photons"], first=x["first"])
             for x in spec.instances]
    total = sum(x.n_photons for x in insts)
    # plain form
    plain_ms, plain_det = 0.0, []
    for x in insts[:2]:                      # warm-up of every context's first launch
        sims[x.context].set_media(x.nmuasg)
        sims[x.context].run(1000, 0)
    t0 = time.perf_counter()
    for x in insts:
        s = sims[x.context]
        s.set_media(x.nmuasg)
        s.zero()
        s.run(x.n_photons, x.first)
        plain_ms += s.kernel_ms()
        plain_det.append(s.tallies()["det"] if len(plain_det) < 4 else None)
    plain_wall = time.perf_counter() - t0
    # batched form
    b = Batch(sims)
    b.set_instances(insts)
    n_own = b.plain_count()
    best, ns = b.autotune(min(total, 8_000_000))
    b.run()                                  # graph capture + first replay
    runs = []
    for _ in range(2):
        t0 = time.perf_counter()
        b.run()
        runs.append((b.last_ms(), time.perf_counter() - t0))
    batch_ms = min(r[0] for r in runs)
    identical = all(np.array_equal(b.tallies(i)["det"], plain_det[i]) for i in range(min(4, len(insts))))
    sig, rel = b.ring_signals()
    from lightpropagation_b200.batch import config_table
    cfg = config_table()[best]
    out = {"instances": len(insts), "meshes": len(spec.meshes),
           "triangles": [int(m.n_tri) for m in spec.meshes], "photons": int(total),
           "budget_range": [args.batch_min, args.batch_max],
           "plain_photons_per_s": total / (plain_ms * 1e-3), "plain_wall_photons_per_s": total / plain_wall,
           "batched_photons_per_s": total / (batch_ms * 1e-3),
           "batched_wall_photons_per_s": total / min(r[1] for r in runs),
           "batched_vs_plain": plain_ms / batch_ms,
           "tallies_identical_to_plain": bool(identical),
           "instances_at_1pct_rse_ring0": int(np.sum(rel[:, 0] <= 0.01)),
           "autotuned_config": cfg, "autotune_ns_per_photon": [float(v) for v in ns],
           "instances_with_own_launch": int(n_own),
           "note": ("plain = device time of one launch per instance; batched = device time of one graph "
                    "launch, which zeroes all instance tallies, runs every instance of at least 2^20 photons "
                    "as a persistent launch of its own and the rest as one persistent batch launch"
                    + ("" if args.batch_min >= 1e6 else
                       "; budgets scaled from the workload's 1e6-1e8 to keep the bench within minutes"))}
    b.close()
    for s in sims:
        s.close()
    return out


def deposits_per_photon(c, n):
    """Fixed-point atomic deposits per photon the transport makes (the algorithmic count):
    per scatter event the r-z cell's absorbed weight and absorbed weight over mua and the
    voxel, less those outside their grids; per photon its exit record's image bins."""
    es = c["scatter"]
    return (2.0 * (es - c["rz_drop"]) + (es - c["vox_drop"])) / n + 10.0


def slab_section(args, local, peak):
    """The same physics on both sides: the 3-layer slab (32 triangles), a pencil beam and
    the reference behaviours on, 1e6 photons per launch.  GPU: device time of 5 launches
    and e2e through the public API; reference: its kernel source on all host cores."""
    from lightpropagation_b200 import Simulation, workloads
    w = workloads.plain_slab()
    n = w.n_photons
    sim = Simulation(local)
    w.apply(sim, seed=0x4C50)
    for i in range(3):
        sim.zero()
        sim.run(n, i * n)
    ms = []
    for i in range(5):
        sim.zero()
        sim.run(n, (3 + i) * n)
        ms.append(sim.kernel_ms())
    t0 = time.perf_counter()
    for i in range(3):
        w.apply(sim, seed=0x4C50 + 7 + i)
        sim.zero()
        sim.run(n, i * n)
        sim.tallies()
    e2e = 3 * n / (time.perf_counter() - t0)
    cnt = sim.tallies()["counters"]
    sim.close()
    out = {"workload": w.name, "photons_per_launch": n, "gpu_photons_per_s": n / (statistics.mean(ms) * 1e-3),
           "gpu_e2e_photons_per_s": e2e, "gpu_events_per_photon": {"scatter": cnt["scatter"] / n,
                                                                  "boundary": cnt["boundary"] / n}}
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        L, why = reference_lib()
        if L is None:
            out["reference_unavailable"] = why
        else:
            m = reference_sample_size([w], threads, 10.0)
            dt, k = reference_sample([w], m, threads)
            out["reference_photons_per_s"] = k / dt
            out["reference_sample"] = f"{k} photons on {threads} threads ({cpu_model()})"
            out["gpu_vs_reference"] = out["gpu_photons_per_s"] / out["reference_photons_per_s"]
            out["gpu_e2e_vs_reference"] = e2e / out["reference_photons_per_s"]
    out["same_physics"] = "pencil beam, reference behaviours Q3/Q4/Q10 on, on both sides"
    return out


def ours_arm(args, cases):
    import torch
    rank, world, local = env_int("RANK", 0), env_int("WORLD_SIZE", 1), env_int("LOCAL_RANK", 0)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
    from lightpropagation_b200 import Simulation, sharding
    from lightpropagation_b200.propagation import fp32_peak_tflops, l2_atomic_peak
    w, ncase = cases[0], len(cases)
    n = w.n_photons
    sim = Simulation(local)
    w.apply(sim, seed=0x4C50)

    red = []
    if dist is not None:
        sim.run(0)                      # allocates the tallies; the aliases stay valid
        red = sharding.device_tally_tensors(sim, local)

    kernel_ms = []          # per timed launch: (case index, device ms)
    last = {}               # each case's tallies after its last timed launch

    def step(i, timed=False):
        """Step i: one launch of n photons (per rank) of case i % ncase.  Returns the
        device ms of the launch plus the all-reduce."""
        j = i % ncase
        c = cases[j]
        if ncase > 1:
            sim.set_media(c.nmuasg)
        sim.zero()
        first, count = sharding.photon_range(n * world, rank, world, i * n * world)
        sim.run(count, first)
        ms = sim.kernel_ms()
        if timed:
            kernel_ms.append((j, ms))
        if dist is not None:
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            sharding.allreduce_flat(red)
            ev1.record()
            ev1.synchronize()
            ms += ev0.elapsed_time(ev1)
        return ms, j

    for i in range(args.warmup):
        step(i)
    # the L2 flush buffer is allocated after the context's own buffers: on this driver a
    # 252 MB block allocated first placed them where the transport kernel ran 15% slower
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.float32, device=f"cuda:{local}")
    peak = fp32_peak_tflops(local)
    atom_peak = l2_atomic_peak(local)
    clocks = ClockSampler(local)
    clocks.start()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    wall0 = time.perf_counter()
    dev_ms = 0.0
    for i in range(args.steps):
        flush.fill_(float(i))           # rewrite a 2x-L2 buffer between timed steps
        torch.cuda.synchronize()
        ms, j = step(args.warmup + i, timed=True)
        dev_ms += ms
        if i >= args.steps - ncase:
            last[j] = sim.tallies()     # after the launch's timing; not part of dev_ms
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

    # gradient cost: one differentiated launch per case (adjoint sums of d(ring signal) /
    # d(mua, mus) for every region) against the mean plain launch of the timed steps
    gradient = None
    if rank == 0 and not args.no_gradient and sim._rings.shape[0] and cases[0].nmuasg.shape[0] <= 8:
        grad_ms, plain_ms = 0.0, 0.0
        for j, c in enumerate(cases):
            ms_j = [k for jj, k in kernel_ms if jj == j]
            if not ms_j:
                continue
            if ncase > 1:
                sim.set_media(c.nmuasg)
            sim.set_gradient(True)
            sim.zero()
            flush.fill_(0.0)
            sim.run(n, 10 ** 12 + j * n)
            grad_ms += sim.kernel_ms()
            sim.set_gradient(False)
            plain_ms += sum(ms_j) / len(ms_j)
        gradient = {"cost_vs_forward": grad_ms / plain_ms, "grad_launch_ms": grad_ms / ncase,
                    "forward_launch_ms": plain_ms / ncase,
                    "derivatives": int(sim._rings.shape[0] * (cases[0].nmuasg.shape[0] - 1) * 2 * ncase),
                    "what": "one launch per case giving d(ring signal)/d(mua, mus) of every region and ring"}

    # e2e through the public API with host buffers, one step per timed step, on the
    # long-lived context of the timed steps (as the reference's CalculatePropagation object
    # is long-lived): every step sets the mesh (BVH build, then upload and cell-grid build
    # at the next run) and the other inputs from host arrays, sets the step's media, runs
    # and copies all tallies back.  Creating and releasing a context stays outside: the
    # release of a context's buffers took 0.005-2 s on this driver, and the same launch
    # ran up to 30 % slower in a context whose buffers the driver placed after other
    # large allocations.  transport_ms_per_step is the device time of the step's launch.
    e2e_v = h2d = d2h = e2e_dev_ms = None
    e2e_steps = args.steps
    if rank == 0 or world > 1:
        e2e_t, e2e_dev_ms, h2d, d2h = 0.0, 0.0, 0, 0
        for i in range(e2e_steps):
            c = cases[i % ncase]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            c.apply(sim, seed=0x4C50 + 1 + i)
            sim.zero()
            sim.run(n, (rank * e2e_steps + i) * n)
            h2d += sim.stats()["h2d_bytes"]
            sim.tallies()
            d2h += sim.stats()["d2h_bytes"]
            e2e_dev_ms += sim.kernel_ms()
            e2e_t += time.perf_counter() - t0
        e2e_v = n * world * e2e_steps / e2e_t
        e2e_dev_ms /= e2e_steps
        h2d //= e2e_steps
        d2h //= e2e_steps
    if dist is None:
        # the batched section's contexts are allocated after this one is released
        sim.close()
        sim = None
        del flush
        torch.cuda.empty_cache()

    if dist is not None:
        red.clear()
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        if sim is not None:
            sim.close()
        return 0

    # roofline of the transport kernel (counters are global after the all-reduce)
    per_launch_photons = n * world
    flops, launch_ms, events, deposits = 0.0, 0.0, {}, 0.0
    rse = {}
    for j, c in enumerate(cases):
        if j not in last:
            continue
        cnt = last[j]["counters"]
        F, es, eb, eq = fp32_flops_per_photon(cnt, per_launch_photons)
        ms_j = [k for jj, k in kernel_ms if jj == j]
        flops += F * n * len(ms_j)
        deposits += deposits_per_photon(cnt, per_launch_photons) * n * len(ms_j)
        launch_ms += sum(ms_j)
        events[c.name] = {"flops_per_photon": F, "scatter": es, "boundary": eb, "query": eq,
                          "query_executed": cnt["query"] / per_launch_photons,
                          "query_skipped_by_safety_bounds": cnt["safe_skip"] / per_launch_photons,
                          "bvh_queries": cnt["bvh_query"] / per_launch_photons,
                          "deposits_per_photon": deposits_per_photon(cnt, per_launch_photons),
                          "avg_launch_ms": sum(ms_j) / len(ms_j), "launches": len(ms_j)}
        det = last[j]["det"]
        if det.shape[0]:
            r = ring_rse(det, per_launch_photons)
            k = sum(1 for jj, _ in kernel_ms if jj == j) * per_launch_photons
            rse[c.name] = {"ring_rse_per_launch": [float(x) for x in r],
                           "ring_rse_over_the_job": [float(x) * float(np.sqrt(per_launch_photons / k)) for x in r],
                           "job_photons": int(k),
                           "photons_for_1pct_rse_at_farthest_ring": float(per_launch_photons * (r[-1] / 0.01) ** 2)}
    achieved = flops / (launch_ms * 1e-3) / 1e12
    atom_rate = deposits / (launch_ms * 1e-3)
    traffic, traffic_photons = traffic_of(args.workload)
    roof = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if peak else None,
            "traffic": (traffic * n / traffic_photons) if traffic is not None else None,
            "traffic_note": (f"dram__bytes_read.sum + dram__bytes_write.sum of one {traffic_photons}-photon 660 nm "
                             f"launch of this workload (ncu, profiles/), scaled to {n} photons")
            if traffic is not None else None,
            "peak_source": "FP32 FMA peak measured in-run by lp_fp32_peak (MEASURED_PEAKS.json has no FP32 figure)",
            "l2_atomics": {"achieved_per_s": atom_rate, "peak_per_s": atom_peak,
                           "frac": atom_rate / atom_peak if atom_peak else None,
                           "what": "64-bit fixed-point deposits (r-z, voxel, exit bins) per second over the rate "
                                   "lp_l2_atomic_peak measures in-run"},
            "events_per_photon": events}

    batched = None
    if world == 1 and args.batch_instances > 0:
        batched = batched_section(args, local)

    slab = None
    if world == 1 and args.workload == "curved_abdomen" and not args.no_slab:
        slab = slab_section(args, local, peak)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            m = reference_sample_size(cases, threads, 12.0)
            dt, k = reference_sample(cases, m, threads)
            cpu = {"value": k / dt, "unit": "photons/s", "cores": threads, "cpu_model": cpu_model(),
                   "kind": "reference",
                   "sample": f"{m} photons of each case of {workload_label(args, cases)}: the reference kernel "
                             f"source compiled for the CPU (oracle/_ref, pencil beam source, brute-force triangle "
                             f"search) on {threads} threads + ExecKernel's host binning"}
        except Exception as e:  # noqa: BLE001
            cpu = {"value": None, "unit": "photons/s", "cores": 0, "kind": "reference", "sample": f"failed: {e}"}

    line = {"metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": workload_label(args, cases), "photons_per_step_per_gpu": n,
                       "photons_per_launch": n, "triangles": int(w.n_tri),
                       "steps_alternate": [c.name for c in cases],
                       "parallelism": f"photon ranges x{world}" + (" + NCCL all-reduce of tallies" if world > 1 else ""),
                       "l2": "2x L2 buffer rewritten between timed steps",
                       "arithmetic": "fast (FMA contraction, MCML direction cosines)",
                       "grid": st["grid"], "block": st["block"], "bvh_nodes": st["n_nodes"],
                       "bvh_nodes_in_smem": st["nodes_smem"], "tris_in_smem": st["tris_smem"]},
            "wall_s": wall, "clocks": clk, "gpu_launches": args.steps,
            "e2e": {"value": e2e_v, "unit": "photons/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "transport_ms_per_step": e2e_dev_ms, "steps": e2e_steps},
            "detector_error": rse, "gradient": gradient, "batched": batched, "config1_slab": slab,
            "roofline": roof, "cpu_baseline": cpu}
    print(json.dumps(line))
    if sim is not None:
        sim.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="curved_abdomen",
                    help="curved_abdomen (660 + 940 nm per step), plain_slab, or another named workload")
    ap.add_argument("--photons", type=int, default=0,
                    help="photons per launch per GPU (default: the workload's, 1e8 for the abdomen)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gradient", action="store_true", help="skip the gradient-cost launches")
    ap.add_argument("--no-slab", action="store_true", help="skip the like-for-like config-1 slab section")
    ap.add_argument("--batch-instances", type=int, default=512, help="instances of the plain-vs-batched "
                    "comparison (0 skips it)")
    ap.add_argument("--batch-min", type=float, default=1e4, help="smallest instance photon budget")
    ap.add_argument("--batch-max", type=float, default=1e6, help="largest instance photon budget")
    args = ap.parse_args()
    cases = load_cases(args.workload, args.photons)
    if args.impl == "reference":
        return reference_arm(args, cases)
    return ours_arm(args, cases)


if __name__ == "__main__":
    sys.exit(main())
