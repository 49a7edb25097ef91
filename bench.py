#!/usr/bin/env python
"""Benchmark: batched Monte Carlo brick-beam solves/s at relative residual 1e-8.

Workload (one step): the uneven Monte Carlo batch -- brick beams 8 x 2 x 2 m
at 20x5x5, 40x10x10 and 60x15x15 elements (2,268 / 14,883 / 46,848 DOFs),
512 samples each, all in one launch.  Per-element E = 30 GPa * exp(0.15 z -
0.01125), z iid N(0,1); nu = 0.2; end-face traction magnitude U(0.8, 1.2) MPa
lumped to the tip nodes; x = 0 face fixed.  Seeded Philox streams per (mesh,
sample), synthetic data.  Every sample is solved to true relative residual
|f - K u| / |f| <= 1e-8 by FP32 Jacobi PCG inside FP64 iterative refinement,
with batched FP64 assembly from unit-E element matrices, and the outputs
(tip displacements, support reactions) are produced on the GPU.

  python bench.py [--gpus N] [--steps K] [--warmup W]     # this implementation
  python bench.py --impl reference [...]                  # the reference, host cores

Multi-GPU (torchrun, one rank per GPU): every rank solves its own 512-sample
batches (weak scaling, no collective on the data path); the step time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MESHES = [(20, 5, 5), (40, 10, 10), (60, 15, 15)]
NSAMP = 512
METRIC = "MC solves/s at rel-res 1e-8: learned+FP32/FP64 batched vs plain FP64 PCG, 1 B200"
WORKLOAD = "MC brick beams 20x5x5 + 40x10x10 + 60x15x15, 512 samples each, one launch"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nsamp", type=int, default=NSAMP)
    p.add_argument("--plain-samples", type=int, default=16, help="samples per mesh timed by the plain method")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiler runs)")
    p.add_argument("--precision", type=int, default=1,
                   help="1: FP32 PCG with FP64 solution and residual replacement; 0: FP64 PCG")
    p.add_argument("--ref-worker", nargs="*", help=argparse.SUPPRESS)
    p.add_argument("--profile-case", action="store_true",
                   help="one small bounded batch (60x15x15, 128 samples, 40 PCG iterations) for ncu captures")
    return p.parse_args()


def profile_case():
    """A bounded case of the same kernels for profiler captures: the 60x15x15
    mesh, 128 samples (values 1.76 GB FP32 > L2), the inner PCG capped at 40
    iterations and one refinement step, run twice (warm + captured)."""
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    from ufem_b200 import meshgen as mg
    m = mg.beam_brick(60, 15, 15, 8.0, 2.0, 2.0, per_element_material=True)
    mg.mc_attach_vars(m)
    f = mg.mc_samples(m, mesh_id=2, nsamp=128)
    g = GpuModel(m)
    for _ in range(2):
        res, st = mc_solve([g], [f], max_iters=40)
    print(json.dumps({"profile_case": "60x15x15 x 128 samples, 40 iterations", "pcg_ms": st.ms_pcg,
                      "pcg_bytes": st.pcg_bytes, "pcg_iterations": st.pcg_iterations,
                      "achieved_GBs": st.pcg_bytes / st.ms_pcg / 1e6 if st.ms_pcg else None}))


def build_meshes(nsamp, rank=0):
    from ufem_b200 import meshgen as mg
    models, iflds = [], []
    for k, (nx, ny, nz) in enumerate(MESHES):
        m = mg.beam_brick(nx, ny, nz, 8.0, 2.0, 2.0, per_element_material=True)
        mg.mc_attach_vars(m, n_out_nodes=4)
        models.append(m)
        iflds.append(mg.mc_samples(m, mesh_id=k, nsamp=nsamp, first_sample=rank * nsamp))
    return models, iflds


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, path):
        self.path = path
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self, device_index=0):
        sm, mx, reasons = [], 0.0, set()
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9 or parts[0] != str(device_index):
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = max(mx, float(parts[2]))
                except ValueError:
                    continue
                names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        except FileNotFoundError:
            pass
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# the reference (host cores): libfem.so's monte_solution, built from the
# reference sources into oracle/_ref; the oracle restatement when absent
# ---------------------------------------------------------------------------
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "thr", "libfem_ref.so")


def ref_worker(args):
    """One process: monte_init_lib_stuff + monte_solution over its samples
    (the reference's own MC solver path, femEqsCGwSSOR, fem/fem_mont.c:498)."""
    import ctypes as C
    import numpy as np
    path, ifld_path, first, count = args[0], args[1], int(args[2]), int(args[3])
    ifld = np.load(ifld_path)
    lib = C.CDLL(REF_LIB)
    lib.monte_init_lib_stuff.argtypes = [C.c_char_p]
    lib.monte_solution.argtypes = [C.c_char_p, C.c_void_p, C.c_void_p, C.c_long]
    lib.monte_nums_of_vars.argtypes = [C.c_char_p] + [C.POINTER(C.c_long)] * 3
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 2)  # the reference prints progress messages
    os.dup2(devnull, 1)
    assert lib.monte_init_lib_stuff(path.encode()) == 0
    il, ol, ff = C.c_long(), C.c_long(), C.c_long()
    lib.monte_nums_of_vars(path.encode(), C.byref(il), C.byref(ol), C.byref(ff))
    out = np.zeros(max(1, ol.value))
    t0 = time.perf_counter()
    for s in range(first, first + count):
        row = np.ascontiguousarray(ifld[s])
        lib.monte_solution(path.encode(), row.ctypes.data, out.ctypes.data, 0)
    dt = time.perf_counter() - t0
    with open(args[4], "w") as f:
        f.write(f"{dt:.6f}\n")


def ref_files(models, iflds, d):
    import numpy as np
    from ufem_b200 import meshgen as mg
    out = []
    for k, (m, f) in enumerate(zip(models, iflds)):
        p = os.path.join(d, f"mc_{k}.fem")
        mg.write_fem(m, p)
        fp = os.path.join(d, f"ifld_{k}.npy")
        np.save(fp, f)
        out.append((p, fp))
    return out


def run_reference_sample(files, procs, samples_per_proc, d):
    """P processes in parallel, each solving `samples_per_proc` samples of
    every mesh; returns (solves, wall seconds)."""
    t0 = time.perf_counter()
    jobs = []
    for p in range(procs):
        for k, (path, fp) in enumerate(files):
            res = os.path.join(d, f"t_{p}_{k}.txt")
            jobs.append(subprocess.Popen([sys.executable, os.path.abspath(__file__), "--ref-worker", path, fp,
                                          str(p * samples_per_proc), str(samples_per_proc), res]))
    for j in jobs:
        j.wait()
    wall = time.perf_counter() - t0
    return procs * samples_per_proc * len(files), wall


def cpu_kind():
    return "reference" if os.path.exists(REF_LIB) else "port"


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def reference_arm(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/thr/libfem_ref.so missing"}))
        return
    models, iflds = build_meshes(max(a.nsamp, 64))
    procs = host_cores()
    with tempfile.TemporaryDirectory() as d:
        files = ref_files(models, iflds, d)
        for _ in range(a.warmup):
            run_reference_sample(files[:1], 1, 1, d)
        times = []
        solves = 0
        for _ in range(a.steps):
            n, wall = run_reference_sample(files, procs, 1, d)
            solves += n
            times.append(wall)
    tot = sum(times)
    value = solves / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000 * tot / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "reference monte_solution (SSOR PCG, eps 1e-21)",
                       "processes": procs},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                             "sample": f"per step: {procs} processes x 1 sample of each of the 3 meshes"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# this implementation
# ---------------------------------------------------------------------------
def ours(a):
    import ctypes as C
    import numpy as np
    import torch
    import torch.distributed as dist
    from ufem_b200 import _lib
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import default_options, mc_solve_serial

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    L = _lib.load()
    models, iflds = build_meshes(a.nsamp, rank)
    gms = [GpuModel(m) for m in models]
    nm = len(gms)
    opt = default_options()
    opt.precision = a.precision
    opt.tol = 1e-8
    dev = torch.device("cuda", local)
    d_in = [torch.from_numpy(f).to(dev) for f in iflds]
    d_out = [torch.zeros((f.shape[0], m.mc_olen), dtype=torch.float64, device=dev) for f, m in zip(iflds, models)]
    d_st = [torch.zeros(f.shape[0], dtype=torch.int32, device=dev) for f in iflds]
    d_it = [torch.zeros(f.shape[0], dtype=torch.int64, device=dev) for f in iflds]
    hs = (C.c_void_p * nm)(*[g.h.value for g in gms])
    ns = np.array([f.shape[0] for f in iflds], np.int64)
    vp = lambda ts: (C.c_void_p * nm)(*[t.data_ptr() for t in ts])
    pin, pout, pst, pit = vp(d_in), vp(d_out), vp(d_st), vp(d_it)
    null = (C.c_void_p * nm)()

    def step_device():
        rv = L.ufem_mc_solve_device(nm, hs, ns.ctypes.data_as(C.POINTER(C.c_long)), pin, pout, pst, pit, null, null,
                                    C.byref(opt))
        _lib.check("ufem_mc_solve_device", rv)

    def barrier():
        if world > 1:
            dist.barrier()

    for _ in range(a.warmup):
        step_device()
    torch.cuda.synchronize()
    stats = _lib.McStats()
    with ClockSampler(os.path.join(tempfile.gettempdir(), f"ufem_clocks_{rank}.csv")) as clk:
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        launches = 0
        pcg_ms = pcg_bytes = spmv_bytes = 0.0
        pcg_launches = pcg_its = 0
        for _ in range(a.steps):
            step_device()
            L.ufem_mc_get_stats(C.byref(stats))
            launches += stats.kernel_launches
            pcg_ms += stats.ms_pcg
            pcg_bytes += stats.pcg_bytes
            spmv_bytes += stats.spmv_bytes
            pcg_launches += stats.pcg_launches
            pcg_its += stats.pcg_iterations
        e1.record()
        torch.cuda.synchronize()
        barrier()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / a.steps
    solves_step = int(ns.sum()) * world
    value = solves_step / (ms_step / 1000.0)
    st_ok = all(bool((s == 0).all()) for s in d_st)
    iters_main = [int(x.max().item()) for x in d_it]
    out_main = d_out[1].cpu().numpy().copy()

    # ---- the other precision, one step, for comparison ----------------------
    alt = None
    if rank == 0:
        opt_main = opt.precision
        opt.precision = 1 - opt_main
        step_device()  # builds its buffers
        torch.cuda.synchronize()
        e0.record()
        step_device()
        e1.record()
        torch.cuda.synchronize()
        alt = {"precision": "FP64 PCG" if opt.precision == 0 else "FP32 PCG + FP64 replacement",
               "value": int(ns.sum()) / (e0.elapsed_time(e1) / 1000.0), "unit": "solves/s",
               "all_converged": all(bool((s == 0).all()) for s in d_st),
               "max_iters_per_mesh": [int(x.max().item()) for x in d_it]}
        opt.precision = opt_main
    iters = iters_main

    # ---- e2e: host (pinned) inputs through the public C ABI call -------------
    h_in = [torch.from_numpy(f).pin_memory() for f in iflds]
    h_out = [torch.zeros((f.shape[0], m.mc_olen), dtype=torch.float64).pin_memory() for f, m in zip(iflds, models)]
    h_st = [torch.zeros(f.shape[0], dtype=torch.int32).pin_memory() for f in iflds]
    h_it = [torch.zeros(f.shape[0], dtype=torch.int64).pin_memory() for f in iflds]
    dp = lambda ts, ty: (C.POINTER(ty) * nm)(*[C.cast(t.data_ptr(), C.POINTER(ty)) for t in ts])
    ein, eout, est, eit = dp(h_in, C.c_double), dp(h_out, C.c_double), dp(h_st, C.c_int), dp(h_it, C.c_long)
    eg = (C.POINTER(C.c_double) * nm)()
    barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        _lib.check("ufem_mc_solve", L.ufem_mc_solve(nm, hs, ns.ctypes.data_as(C.POINTER(C.c_long)), ein, eout, est,
                                                    eit, eg, C.byref(opt)))
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / a.steps
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    h2d = sum(f.nbytes for f in iflds)
    d2h = sum(o.numel() * 8 + s.numel() * 4 + i.numel() * 8 for o, s, i in zip(h_out, h_st, h_it))
    e2e_ok = np.allclose(h_out[1].numpy(), out_main, rtol=1e-12, atol=0)

    result = None
    if rank == 0:
        # ---- the plain method on a subset of the same samples ---------------
        plain_t = 0.0
        plain_n = 0
        plain_its = []
        for g, f in zip(gms, iflds):
            sub = f[:a.plain_samples]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            o, st, it = mc_solve_serial(g, sub, tol=1e-8)
            torch.cuda.synchronize()
            plain_t += (time.perf_counter() - t0) * (f.shape[0] / sub.shape[0])
            plain_n += f.shape[0]
            plain_its.append(int(it.max()))
        plain = plain_n / plain_t
        peak, peak_kind = measured_peaks()
        achieved = pcg_bytes / (pcg_ms / 1000.0) / 1e9 if pcg_ms > 0 else 0.0
        # DRAM traffic per launch: the ncu-measured traffic / algorithmic
        # ratio of this kernel (profiles/, a smaller case of the same kernel)
        # times this run's algorithmic bytes per launch
        traffic = None
        tf = os.path.join(ROOT, "profiles", "k_batch_pcg_60x15x15_128samples.md")
        if os.path.exists(tf) and pcg_launches > 0:
            for line in open(tf):
                if line.startswith("traffic_over_algorithmic:"):
                    traffic = float(line.split(":")[1]) * pcg_bytes / pcg_launches
        # ---- CPU baseline: the reference on a bounded sample ------------------
        cpu = None
        if os.path.exists(REF_LIB) and not a.no_cpu:
            procs = host_cores()
            with tempfile.TemporaryDirectory() as d:
                files = ref_files(models, [f[:max(1, procs)] for f in iflds], d)
                n, wall = run_reference_sample(files, procs, 1, d)
            cpu = {"value": n / wall, "unit": "solves/s", "cores": procs, "kind": "reference",
                   "sample": f"{procs} processes x 1 sample of each mesh via monte_solution ({wall:.1f} s)"}
        result = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 inner / fp64 refinement", "data": "synthetic",
            "config": {"workload": WORKLOAD, "samples_per_step": solves_step, "rel_res": 1e-8,
                       "precision": "FP32 Jacobi PCG in FP64 iterative refinement",
                       "l2_flush": "not needed: batched values 9.5 GB per iteration >> 126 MB L2",
                       "parallelism": f"samples sharded over {world} GPU(s), no collective"},
            "all_converged": st_ok, "max_iters_per_mesh": iters,
            "plain_fp64_one_at_a_time": {"value": plain, "unit": "solves/s", "max_iters_per_mesh": plain_its,
                                         "samples_timed_per_mesh": a.plain_samples},
            "speedup_vs_plain": value / plain,
            "roofline": {"bound": "hbm", "kernel": "k_batch_pcg<float,3>", "achieved": achieved,
                         "peak": peak, "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "pcg_ms_per_step": pcg_ms / a.steps,
                         "pcg_launches_per_step": pcg_launches / a.steps,
                         "pcg_iterations_per_step": pcg_its / a.steps},
            "e2e": {"value": solves_step / (e2e_ms / 1000.0), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "matches_device_run": bool(e2e_ok)},
            "gpu_launches": launches, "clocks": clk.summary(local), "other_precision": alt,
            "cpu_baseline": cpu,
        }
        print(json.dumps(result))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.ref_worker:
        ref_worker(a.ref_worker)
        return
    if a.profile_case:
        profile_case()
        return
    if a.impl == "reference":
        reference_arm(a)
    else:
        ours(a)


if __name__ == "__main__":
    main()
