#!/usr/bin/env python
"""Benchmark: Monte Carlo brick-beam solves/s at relative residual 1e-8,
learned warm start + batched PCG against plain FP64 PCG, 1 B200.

Workload (one step): 8,192 fresh samples of the 40x10x10 brick cantilever
beam (8 x 2 x 2 m, 14,883 DOFs) with 16 equal-length E zones along x
(E = 30 GPa * exp(0.15 z), z iid N(0,1), median 30 GPa) and one load factor
U(0.8, 1.2) on the 1 MPa end-face traction (17 random inputs), x = 0 face
fixed, seeded Philox streams per sample, synthetic data.

Set-up (not timed): 4,096 training samples solved by the batched solver, a
64-mode POD basis from the first 512 solutions, the per-zone reduced
operators Phi^T K_z Phi, and a 17-256-256-64 GELU MLP trained on the tensor
cores (CUDA-graph-replayed steps).

Timed step (ufem_warm_solve): the guess -- by default each sample's
POD-Galerkin coefficients on the learned basis (--guess 1), or the MLP's
coefficients (--guess 0) -- then the batched Jacobi PCG to |f - K u| / |f|
<= 1e-8 for every sample, by default in FP64 with every 3x3 block formed in
the kernel from the shared unit-E element blocks (--precision 2; 1 = FP32
PCG on explicit FP32 matrices with FP64 solution and true-residual
replacement, 0 = explicit FP64), cold fallback for samples whose iterations
regress, outputs (tip displacements, reactions) on the GPU.

Reported beside it: the other guess, the other precisions, the same batch
without a warm start, the plain method (FP64 assembly + FP64 Jacobi PCG, one
sample at a time, on a subset of the same samples), the uneven batch
(20x5x5 + 40x10x10 + 60x15x15 beams, per-element lognormal E, 512 samples
each, one launch), the single-system configs (80x20x20 beam, 128x128x64
block; FP64 and FP32-inner/FP64-refinement PCG) and the reference's own
Monte Carlo library on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W]     # this implementation
  python bench.py --impl reference [...]                  # the reference, host cores

Multi-GPU (torchrun, one rank per GPU): every rank trains the same warm start
and solves its own 8,192 samples (weak scaling, no collective on the data
path); the step time is the max over ranks.
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

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MESHES = [(20, 5, 5), (40, 10, 10), (60, 15, 15)]
NSAMP = 512
WARM_MESH = (40, 10, 10)
WARM_ZONES = 16
WARM_TRAIN = 4096
WARM_EVAL = 8192
EVAL_FIRST = 1 << 20     # evaluation sample ids: disjoint from training
METRIC = "MC solves/s at rel-res 1e-8: learned+FP32/FP64 batched vs plain FP64 PCG, 1 B200"
WORKLOAD = ("MC 40x10x10 brick beam, 16 lognormal E zones + load factor (17 inputs), 8192 fresh samples "
            "warm-started by the learned guess (POD 64 modes from 512 solves; least-squares quadratic model of the "
            "POD coefficients in the zone compliances 1/E + MLP 17-256-256-64 on its residual, trained on 4096 "
            "solves) and solved by FP32 PCG with FP64 solution and true-residual replacement, preconditioner "
            "coarse-corrected on {c} POD modes of the same snapshots")
UNEVEN = "MC brick beams 20x5x5 + 40x10x10 + 60x15x15, 512 samples each, one launch"
KERNEL = {0: "k_batch_pcg<double,3,explicit>", 1: "k_batch_pcg<float,3,explicit>",
          2: "k_batch_pcg<double,3,implicit>", 3: "k_batch_pcg<float,3,implicit>",
          4: "k_batch_pcg<float,3,implicit,fp32 products>"}
# precision 4 with the coarse space: each iteration is a k_batch_s launch (q = A z) and a k_batch_pcg launch
KERNEL_SPLIT = "k_batch_s<float,3,fp32 products> (q = A z) + k_batch_pcg<float,3,implicit,fp32 products> (updates, true residuals, tcgen05 coarse phases), one pair of launches per iteration"
PREC = {0: "FP64 PCG, explicit FP64 matrix per sample",
        1: "FP32 PCG on explicit FP32 matrices, FP64 solution and true-residual replacement",
        2: "FP64 PCG, blocks formed in the kernel from shared unit-E element blocks",
        3: "FP32 PCG (FP32 vectors, FP64 products of blocks formed in the kernel from the unit-E blocks), "
           "FP64 solution and FP64 true-residual replacement",
        4: "FP32 PCG (FP32 vectors and FP32 SpMV products: blocks formed in the kernel from FP32 copies of the "
           "unit-E blocks), FP64 solution and FP64 true-residual replacement"}
GUESS = {0: "learned: least-squares quadratic model + MLP (BF16 tcgen05 network) of the POD coefficients",
         1: "each sample's POD-Galerkin coefficients (Phi^T K_s Phi c = Phi^T f_s) on the learned POD basis",
         2: "the least-squares quadratic model alone (no network)"}
EPS_ORACLE = 1e-17 / 10000.0  # the reference's stopping rule, FEM_ZERO/10000 (fem/fem.h:59, fem/fem_sol.c:1722)
FP64_NOMINAL_TFLOPS = 37.0   # B200 FP64 (non-tensor) peak, datasheet figure: not measured here
BRICK_FLOP = 2.3e5           # FP64 flops of the reference's 27-point brick integration per element


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--nsamp", type=int, default=NSAMP, help="samples per mesh of the uneven batch")
    p.add_argument("--train", type=int, default=WARM_TRAIN, help="warm-start training samples")
    p.add_argument("--eval", type=int, default=WARM_EVAL, help="warm-started samples per step and rank")
    p.add_argument("--epochs", type=int, default=100, help="MLP training epochs")
    p.add_argument("--plain-samples", type=int, default=16, help="samples timed by the plain method")
    p.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch section")
    p.add_argument("--no-other", action="store_true", help="skip the other precisions of the warm start")
    p.add_argument("--no-coarse", action="store_true",
                   help="headline without the coarse correction of the preconditioner (Jacobi PCG)")
    p.add_argument("--coarse-modes", type=int, default=128,
                   help="POD modes of the preconditioner's coarse space (a multiple of 16, at most 128); the "
                        "guess and the MLP use the 64-mode basis of the learned-warm-start config")
    p.add_argument("--no-static", action="store_true", help="skip the single-system configs (80x20x20, 128x128x64)")
    p.add_argument("--tiles-per-block", type=int, default=0, help=argparse.SUPPRESS)
    p.add_argument("--guess", type=int, default=0,
                   help="warm-start guess: 0 = the learned coefficients (least-squares model + MLP, default), "
                        "1 = each sample's POD-Galerkin coefficients on the learned basis, 2 = the least-squares "
                        "model alone")
    p.add_argument("--precision", type=int, default=4,
                   help="4: FP32 PCG with FP32 SpMV products, FP64 solution and true-residual replacement, blocks "
                        "formed in the kernel (default); 3: the same with FP64 products; 2: FP64 PCG, blocks formed "
                        "in the kernel; 1: FP32 PCG on explicit FP32 matrices; 0: FP64 explicit")
    p.add_argument("--oracle-samples", type=int, default=64,
                   help="evaluation samples checked against the FP64 oracle (displacements, von Mises)")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline (profiler runs)")
    p.add_argument("--ref-worker", nargs="*", help=argparse.SUPPRESS)
    p.add_argument("--profile-case", action="store_true",
                   help="one small bounded batch (60x15x15, 128 samples, 40 PCG iterations) for ncu captures")
    p.add_argument("--profile-samples", type=int, default=1024,
                   help="samples of the --profile-case batch (precisions 2 and 3: the 40x10x10 zone beam)")
    p.add_argument("--profile-static", action="store_true",
                   help="the 128x128x64 block's FP64 PCG capped at 40 iterations (two launches) for ncu captures")
    p.add_argument("--profile-ingest", action="store_true",
                   help="input-file ingest of the 128x128x64 block: text vs binary form (host parse, then the "
                        "whole ufem_read_input with the model build and upload)")
    p.add_argument("--profile-outputs", type=int, default=0, metavar="SAMPLES",
                   help="the Monte Carlo output pass (element sums/extremes, RES_E, RES_FAIL) on the 40x10x10 "
                        "zone beam with SAMPLES samples, against the same batch with RES_D/RES_R only")
    return p.parse_args()


PROFILE = {1: ("k_batch_pcg_60x15x15_128samples.md", "60x15x15 per-element E x 128 samples, 40 iterations"),
           4: ("k_batch_split_fp32prod_coarse_40x10x10_4096samples.md",
               "40x10x10 16 E zones, FP32 implicit form with FP32 products, coarse space and learned guess of a "
               "short warm-start training, PCG to 1e-8"),
           3: ("k_batch_pcg_fp32_coarse_40x10x10_2048samples.md",
               "40x10x10 16 E zones x 2048 samples, FP32 implicit form, coarse space of a short warm-start "
               "training, 40 iterations"),
           2: ("k_batch_pcg_coarse_40x10x10_1024samples.md",
               "40x10x10 16 E zones x 1024 samples, coarse space of a short warm-start training, 40 iterations")}


def profile_case(a):
    """A bounded case of the same kernels for profiler captures, run twice
    (warm + captured), the inner PCG capped at 40 iterations.  Precision 1:
    the 60x15x15 per-element-E beam, 128 samples (FP32 values 1.76 GB > L2);
    precision 2: the 40x10x10 zone beam, 1,024 samples (every FP64 vector
    122 MB, eight of them > L2)."""
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    from ufem_b200 import meshgen as mg
    if a.precision in (2, 3, 4):
        m = mg.warm_beam(*WARM_MESH, zones=WARM_ZONES)
        f = mg.warm_samples(m, a.profile_samples)
        if not a.no_coarse:
            # the coarse space from a short warm-start training (sets it on the model)
            from ufem_b200.warm import WarmStart
            g = GpuModel(m)
            cols, logs, scale_col = mg.warm_features(m)
            ws = WarmStart(g, cols, logs, scale_col, n_modes=64, n_hidden=64, n_snapshots=512, epochs=2,
                           batch=256, n_coarse=a.coarse_modes)
            ws.train(mg.warm_samples(m, 1024, first_sample=EVAL_FIRST), precision=2)
    else:
        m = mg.beam_brick(60, 15, 15, 8.0, 2.0, 2.0, per_element_material=True)
        mg.mc_attach_vars(m)
        f = mg.mc_samples(m, mesh_id=2, nsamp=128)
    if a.precision not in (2, 3, 4) or a.no_coarse:
        g = GpuModel(m)
    if a.precision == 4 and not a.no_coarse:
        # precision 4 (FP32 products) runs warm-started only: the short
        # training's learned guess, the PCG to 1e-8
        import ctypes as C
        from ufem_b200 import _lib
        for _ in range(2):
            ws.solve(f, precision=4, tiles_per_block=a.tiles_per_block)
        st = _lib.McStats()
        _lib.load().ufem_mc_get_stats(C.byref(st))
    else:
        for _ in range(2):
            res, st = mc_solve([g], [f], precision=a.precision, max_iters=40, tiles_per_block=a.tiles_per_block,
                               coarse=0 if a.no_coarse else 1)
    print(json.dumps({"profile_case": PROFILE.get(a.precision, ("", ""))[1], "coarse_modes": st.coarse_modes,
                      "pcg_ms": st.ms_pcg,
                      "pcg_bytes": st.pcg_bytes, "pcg_iterations": st.pcg_iterations,
                      "achieved_GBs": st.pcg_bytes / st.ms_pcg / 1e6 if st.ms_pcg else None,
                      "phase_wall_ms": list(st.phase_wall_ms), "phase_busy_ms": list(st.phase_busy_ms)}))


def profile_static(a):
    """A bounded case of the single-system FP64 PCG (`k_cg`) for profiler
    captures: the 128x128x64 block (3,244,995 DOFs, 2.1 GB of FP64 block
    values, ~2.3 GB on the device), two launches capped at 40 iterations."""
    import ctypes as C
    import numpy as np
    from ufem_b200 import _lib, api, meshgen as mg
    from ufem_b200.api import GpuModel
    m = mg.block_brick(128, 128, 64)
    g = GpuModel(m)
    g.fill_K(0)
    g.add_loads()
    g.add_disps()
    L = _lib.load()
    b, nbr, nnzb = g.bsr_shape()
    n = g.ndof
    sol_ms, x = C.c_double(), C.c_double()
    for _ in range(2):
        g.set_u(np.zeros(n))
        rv, its = g.solve(api.SOLVER_CGWJ, api.STOP_RELRES, 1e-30, 40, check=False)  # the cap ends it
        L.ufem_get_phase_ms(g.h, C.byref(x), C.byref(x), C.byref(sol_ms), C.byref(x))
    by = its * (nnzb * 76.0 + 4.0 * (nbr + 1) + 13.0 * n * 8)
    print(json.dumps({"profile_static": "128x128x64 block, FP64 PCG, 40 iterations", "iterations": its,
                      "solve_ms": sol_ms.value, "algorithmic_bytes": by,
                      "achieved_GBs": by / sol_ms.value / 1e6 if sol_ms.value else None}))


def profile_outputs(a):
    """The Monte Carlo output pass at the warm-start workload's size: the
    40x10x10 beam with 16 type-5 zones (they hold F_YC), the output table of
    `mc_attach_outputs` (element sums/maxima/minima/fail flags over stresses
    and strains, RES_E points, RES_FAIL with F_YC and MAX_D per sample) and
    the same batch with RES_D/RES_R outputs only; PCG capped at 40
    iterations (the outputs do not depend on the cap), each run twice (warm,
    timed).  The pass reads u twice (element gathers, max |u|), E once, and
    writes and reads one record of 3 x 12 + 1 doubles per (element range,
    sample)."""
    import numpy as np
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import mc_solve
    S = a.profile_outputs
    rows = {}
    for kind in ("plain", "outputs"):
        m = mg.warm_beam(*WARM_MESH, zones=WARM_ZONES)
        m.mp_type = np.full(len(m.mp_vals), mg.MAT_STRENGTH, np.int64)
        m.mp_vals = [np.array([2500.0, 30e9, 0.2, 12.5e9, 24e6, 2e6, 30e6, 2e6]) for _ in m.mp_vals]
        if kind == "plain":
            f = mg.mc_samples(m, mesh_id=4, nsamp=S)
        else:
            mg.mc_attach_outputs(m)
            # stresses of this beam reach ~24 MPa at the support; tip deflection ~1.7 cm
            f = mg.mc_outputs_samples(m, S, vm_scale=24e6, u_scale=0.13)
        g = GpuModel(m)
        for _ in range(2):
            res, st = mc_solve([g], [f], precision=2, max_iters=40, coarse=0)
        rows[kind] = dict(ms_outputs=st.ms_outputs, ms_pcg=st.ms_pcg, launches=st.kernel_launches,
                          olen=m.mc_olen, ne=m.eLen, n=g.ndof)
    n, ne = rows["outputs"]["n"], rows["outputs"]["ne"]
    nch = max(1, min(ne, -(-4 * 148 // (S // 128))))
    by = 2.0 * n * S * 8 + ne * S * 8.0 + 2.0 * nch * 37 * S * 8
    dt = rows["outputs"]["ms_outputs"] - rows["plain"]["ms_outputs"]
    print(json.dumps({"profile_outputs": f"40x10x10 16 type-5 zones x {S} samples", "plain": rows["plain"],
                      "outputs": rows["outputs"], "element_pass_ms": dt, "element_pass_bytes": by,
                      "achieved_GBs": by / dt / 1e6 if dt > 0 else None}))


def profile_ingest(a):
    """Ingest of the 128x128x64 block's input file (1.1 M nodes, 1 M
    elements): `ufem_convert_input` from the text form and from the binary
    form (parse + write of the binary file, host only), then
    `ufem_read_input` of each form (parse, DOF numbering, pattern, upload)."""
    import tempfile
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel, convert_input
    d = tempfile.mkdtemp()
    m = mg.block_brick(128, 128, 64)
    txt, b1, b2 = (os.path.join(d, f) for f in ("block.fem", "block.bin", "block2.bin"))
    mg.write_fem(m, txt)
    t0 = time.perf_counter()
    convert_input(txt, b1)
    t1 = time.perf_counter()
    convert_input(b1, b2)
    t2 = time.perf_counter()
    rd, stages = {}, {}
    for form, path in (("text", txt), ("binary", b1)):
        GpuModel(path=path).close()  # first-call set-up out of the timing
        best = None
        for _ in range(3):
            s0 = time.perf_counter()
            g = GpuModel(path=path)
            t = time.perf_counter() - s0
            if best is None or t < best:
                best, stages[form] = t, {k: round(v, 2) for k, v in g.ingest_ms().items()}
            g.close()
        rd[form] = best
    print(json.dumps({"profile_ingest": "128x128x64 block input file", "text_MB": os.path.getsize(txt) / 1e6,
                      "binary_MB": os.path.getsize(b1) / 1e6, "convert_from_text_s": t1 - t0,
                      "convert_from_binary_s": t2 - t1, "read_input_text_s": rd["text"],
                      "read_input_binary_s": rd["binary"], "stages_ms": stages,
                      "timing": "best of 3 reads each; stages_ms: file read, parse, host tables, DOF numbering + "
                                "pattern + scatter map + colouring (device), supports/loads, upload"}))


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
        # nvidia-smi's start-up (NVML initialisation) must not fall into the
        # timed region: wait for its first sample
        t0 = time.time()
        while self.proc is not None and time.time() - t0 < 5.0:
            try:
                if os.path.getsize(self.path) > 0:
                    break
            except OSError:
                pass
            time.sleep(0.05)
        time.sleep(0.3)
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


def warm_setup(a, rank=0):
    """The warm-start model, its training samples and this rank's evaluation samples."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.shard import rank_samples
    m = mg.warm_beam(*WARM_MESH, zones=WARM_ZONES)
    train = mg.warm_samples(m, a.train)
    first, count = rank_samples(rank, a.eval, EVAL_FIRST)
    ev = mg.warm_samples(m, count, first_sample=first)
    return m, train, ev


def reference_arm(a):
    """The reference's own Monte Carlo library (monte_solution -> femEqsCGwSSOR,
    fem/fem_mont.c:480-508) on the host cores: P processes, each solving its
    share of the warm-start workload's evaluation samples.  Rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref/thr/libfem_ref.so missing"}))
        return
    m, _, ev = warm_setup(argparse.Namespace(train=1, eval=max(64, host_cores())))
    procs = host_cores()
    with tempfile.TemporaryDirectory() as d:
        files = ref_files([m], [ev], d)
        for _ in range(a.warmup):
            run_reference_sample(files, 1, 1, d)
        times, solves = [], 0
        for _ in range(a.steps):
            n, wall = run_reference_sample(files, procs, 1, d)
            solves += n
            times.append(wall)
    tot = sum(times)
    value = solves / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000 * tot / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD.format(c=a.coarse_modes), "solver": "reference monte_solution (SSOR PCG, eps 1e-21)",
                       "processes": procs},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": procs, "kind": "reference",
                             "sample": f"per step: {procs} processes x 1 evaluation sample of the 40x10x10 "
                                       "warm-start beam"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------------------
# this implementation
# ---------------------------------------------------------------------------
def _vp(ts):
    import ctypes as C
    return (C.c_void_p * len(ts))(*[t.data_ptr() for t in ts])


def uneven_section(a, rank, dev):
    """The uneven batch: three meshes, a.nsamp samples each, one launch; one
    warm-up and one timed step, cold starts, for the FP32-inner / FP64
    refinement form (explicit FP32 matrices) and the FP64 implicit form."""
    import ctypes as C
    import numpy as np
    import torch
    from ufem_b200 import _lib
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import default_options
    L = _lib.load()
    models, iflds = build_meshes(a.nsamp, rank)
    gms = [GpuModel(m) for m in models]
    nm = len(gms)
    d_in = [torch.from_numpy(f).to(dev) for f in iflds]
    d_out = [torch.zeros((f.shape[0], m.mc_olen), dtype=torch.float64, device=dev) for f, m in zip(iflds, models)]
    d_st = [torch.zeros(f.shape[0], dtype=torch.int32, device=dev) for f in iflds]
    d_it = [torch.zeros(f.shape[0], dtype=torch.int64, device=dev) for f in iflds]
    hs = (C.c_void_p * nm)(*[g.h.value for g in gms])
    ns = np.array([f.shape[0] for f in iflds], np.int64)
    null = (C.c_void_p * nm)()
    out = {"workload": UNEVEN}
    for prec, label in ((1, "fp32_explicit_fp64_refinement"), (2, "fp64_implicit"), (3, "fp32_implicit_fp64_refinement")):
        opt = default_options()
        opt.precision = prec
        opt.tol = 1e-8
        args = (nm, hs, ns.ctypes.data_as(C.POINTER(C.c_long)), _vp(d_in), _vp(d_out), _vp(d_st), _vp(d_it), null,
                null, C.byref(opt))
        _lib.check("ufem_mc_solve_device", L.ufem_mc_solve_device(*args))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _lib.check("ufem_mc_solve_device", L.ufem_mc_solve_device(*args))
        e1.record()
        torch.cuda.synchronize()
        st = _lib.McStats()
        L.ufem_mc_get_stats(C.byref(st))
        ms = e0.elapsed_time(e1)
        out[label] = {"value": int(ns.sum()) / (ms / 1000.0), "unit": "solves/s", "ms_per_step": ms,
                      "all_converged": all(bool((x == 0).all()) for x in d_st),
                      "max_iters_per_mesh": [int(x.max().item()) for x in d_it],
                      "pcg_GBs": st.pcg_bytes / (st.ms_pcg / 1000.0) / 1e9 if st.ms_pcg else None}
    del gms
    return out


def static_section(a, peak):
    """Configs 2 and 3 of the single-system path: the 80x20x20 brick
    cantilever (107,163 DOFs) and the 128x128x64 block (3,244,995 DOFs), each
    solved to true relative residual 1e-8 by the plain FP64 Jacobi PCG and by
    the FP32-inner / FP64-refinement PCG, with the error of each against a
    FP64 solve to 1e-12.  Bytes are algorithmic (the block-sparse PCG count): one FP64
    PCG iteration reads nb*(72+4) + 4*(nbr+1) + 13*n*8 bytes, one FP32 inner
    iteration nb*(36+4) + 4*(nbr+1) + 13*n*4, one FP64 residual nb*(72+4) +
    4*(nbr+1) + 3*n*8."""
    import ctypes as C
    import numpy as np
    from ufem_b200 import api, meshgen as mg
    from ufem_b200.api import GpuModel
    out = {}
    for name, m in (("beam_80x20x20", mg.beam_brick(80, 20, 20, 8.0, 2.0, 2.0)),
                    ("block_128x128x64", mg.block_brick(128, 128, 64))):
        t0 = time.perf_counter()
        g = GpuModel(m)
        g.fill_K(0)
        g.add_loads()
        g.add_disps()
        setup_s = time.perf_counter() - t0
        # element integration + colour-ordered assembly (fem_fill_K(0)): the
        # second call, CUDA events inside the library
        fills = []
        for _ in range(3):
            g.fill_K(0)
            fills.append(g.phase_ms()["fill"])
        g.add_loads()
        g.add_disps()
        fill_best = min(fills)
        b, nbr, nnzb = g.bsr_shape()
        n = g.ndof
        fill_ms = C.c_double(); bc_ms = C.c_double(); sol_ms = C.c_double(); res_ms = C.c_double()
        L = g.L if hasattr(g, "L") else None
        from ufem_b200 import _lib
        L = _lib.load()
        res = {"ndof": n, "blocks": nnzb, "setup_s": setup_s,
               "fill_K": {"ms": fill_best, "elements": int(m.eLen),
                          "elements_per_s": m.eLen / (fill_best / 1000.0),
                          "reference_equivalent_TFLOPs": m.eLen * BRICK_FLOP / (fill_best / 1000.0) / 1e12,
                          "frac_of_nominal_fp64": m.eLen * BRICK_FLOP / (fill_best / 1000.0) / 1e12
                          / FP64_NOMINAL_TFLOPS,
                          "note": "integration of every brick (closed-form isotropic H^T D H at 27 points) and "
                                  "the colour-ordered scatter into the block-sparse K; FLOPs counted as the "
                                  "reference's 2.3e5 per brick (27 x (H^T D + (H^T D) H)); FP64 peak: the "
                                  "B200 datasheet's 37 TFLOP/s, not measured"}}
        g.set_u(np.zeros(n))
        g.solve(api.SOLVER_CGWJ, api.STOP_RELRES, 1e-12, 0)
        uref = g.u()
        for label, solver in (("fp64", api.SOLVER_CGWJ), ("fp32_fp64_refinement", api.SOLVER_CGWJ_MIXED)):
            g.set_u(np.zeros(n))
            g.solve(solver, api.STOP_RELRES, 1e-8, 0)  # warm-up
            best = None
            for _ in range(2):
                g.set_u(np.zeros(n))
                rv, its = g.solve(solver, api.STOP_RELRES, 1e-8, 0)
                L.ufem_get_phase_ms(g.h, C.byref(fill_ms), C.byref(bc_ms), C.byref(sol_ms), C.byref(res_ms))
                if best is None or sol_ms.value < best[0]:
                    best = (sol_ms.value, its, rv)
            ms, its, rv = best
            u = g.u()
            if solver == api.SOLVER_CGWJ:
                by = its * (nnzb * 76.0 + 4.0 * (nbr + 1) + 13.0 * n * 8)
            else:
                by = its * (nnzb * 40.0 + 4.0 * (nbr + 1) + 13.0 * n * 4)
            res[label] = {"converged": rv == 0, "iterations": its, "ms": ms,
                          "DOF_iterations_per_s": n * its / (ms / 1000.0),
                          "achieved_GBs": by / (ms / 1000.0) / 1e9, "frac_of_measured_hbm": by / (ms / 1000.0) / 1e9 / peak,
                          "u_rel_err_vs_fp64_1e-12": float(np.abs(u - uref).max() / np.abs(uref).max())}
        if name.startswith("beam"):
            # the reference's -nes (BiCGStab) and -ssor (SSOR PCG) solvers on
            # the same system, persistent kernels, to the same 1e-8 residual
            for label, solver in (("bicgstab", api.SOLVER_BICG), ("ssor_pcg", api.SOLVER_SSOR)):
                g.set_u(np.zeros(n))
                g.solve(solver, api.STOP_RELRES, 1e-8, 0, check=False)
                g.set_u(np.zeros(n))
                rv, its = g.solve(solver, api.STOP_RELRES, 1e-8, 0, check=False)
                L.ufem_get_phase_ms(g.h, C.byref(fill_ms), C.byref(bc_ms), C.byref(sol_ms), C.byref(res_ms))
                u = g.u()
                res[label] = {"converged": rv == 0, "iterations": its, "ms": sol_ms.value,
                              "u_rel_err_vs_fp64_1e-12": float(np.abs(u - uref).max() / np.abs(uref).max())}
        out[name] = res
        del g
    return out


def _von_mises(sig):
    """von Mises stress of (SX, SY, SZ, SYZ, SZX, SXY) records."""
    sx, sy, sz, syz, szx, sxy = (sig[..., k] for k in range(6))
    return (0.5 * ((sx - sy) ** 2 + (sy - sz) ** 2 + (sz - sx) ** 2) + 3.0 * (sxy ** 2 + syz ** 2 + szx ** 2)) ** 0.5


def _oracle_job(job):
    """One process of the oracle leg: the samples' static solves by the C
    restatement of the reference (oracle/ufem_oracle.c).  eps > 0: the
    reference's own stopping rule (FEM_ZERO/10000: converged to FP64, the
    checker); eps < 0: the relative residual |eps| (the CPU leg at the GPU's
    tolerance).  Returns per sample (u, von Mises at the brick's stored
    points 1-19, iterations, seconds)."""
    from oracle.oracle import OracleModel
    from ufem_b200 import meshgen as mg
    model, rows, eps, want_fields = job
    out = []
    for row in rows:
        ms = mg.model_for_sample(model, row)
        t0 = time.perf_counter()
        o = OracleModel(ms).run_static(eps=eps)
        dt = time.perf_counter() - t0
        out.append((o["u"] if want_fields else None, _von_mises(o["sig"][:, :19, :]) if want_fields else None,
                    o["iters"], dt, o["rv_solve"]))
    return out


def oracle_leg(model, rows, eps, procs, want_fields=True):
    """The oracle over `rows` in `procs` spawned processes (spawned: this
    process already holds a CUDA context); returns the per-sample results and
    the wall time."""
    import multiprocessing as mp
    chunks = [rows[i::procs] for i in range(procs) if len(rows[i::procs])]
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(len(chunks)) as pool:
        parts = pool.map(_oracle_job, [(model, c, eps, want_fields) for c in chunks])
    wall = time.perf_counter() - t0
    res = [None] * len(rows)
    for i, part in enumerate(parts):
        for j, r in enumerate(part):
            res[i + j * len(chunks)] = r
    return res, wall


def warm_run(L, ws, d, guess, precision, coarse, steps, tol=1e-8):
    """ufem_warm_solve with the given guess, precision and coarse correction:
    one warm-up call, then `steps` timed calls (CUDA events)."""
    import ctypes as C
    import torch
    from ufem_b200 import _lib
    from ufem_b200.mc import default_options
    n = d["in"].shape[0]
    L.ufem_warm_set_guess_mode(ws.h, guess)
    o = default_options()
    o.precision = precision
    o.tol = tol
    o.coarse = int(bool(coarse))
    st = _lib.WarmStats()
    args = (ws.h, n, d["in"].data_ptr(), d["out"].data_ptr(), d["st"].data_ptr(), d["it"].data_ptr(), C.byref(o),
            C.byref(st))
    _lib.check("ufem_warm_solve", L.ufem_warm_solve(*args))
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    pcg_ms = pcg_by = 0.0
    for _ in range(steps):
        _lib.check("ufem_warm_solve", L.ufem_warm_solve(*args))
        pcg_ms += st.pcg_ms
        pcg_by += st.pcg_bytes
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    it = d["it"].cpu().numpy()
    return {"guess": GUESS[guess], "precision": PREC[precision], "coarse": bool(coarse),
            "value": n / (ms / 1000.0), "unit": "solves/s", "ms_per_step": ms, "iters_mean": float(it.mean()),
            "iters_max": int(it.max()), "guess_rel_err_mean": st.guess_err_mean, "guess_rel_err_max": st.guess_err_max,
            "fallbacks": st.fallbacks, "all_converged": bool(np.isin(d["st"].cpu().numpy(), [0, 4]).all()),
            "pcg_GBs": pcg_by / (pcg_ms / 1000.0) / 1e9 if pcg_ms else None}, d["out"].cpu().numpy().copy()


def solve_u(L, g, ws, rows, guess, precision, coarse, tol=1e-8):
    """The displacements of `rows` by the same method (ufem_warm_guess, then
    the batched solve from the guesses), u [nsamp][ndof]."""
    import ctypes as C
    import torch
    from ufem_b200 import _lib
    from ufem_b200.mc import default_options
    L.ufem_warm_set_guess_mode(ws.h, guess)
    u0 = ws.guess(rows)
    n = rows.shape[0]
    S = max(128, (n + 127) // 128 * 128)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    g0 = np.zeros((g.ndof, S))
    g0[:, :n] = u0.T  # the device guess layout: [nDOFAct][S], sample fastest
    d_in, d_g = t(rows), t(g0)
    d_out = torch.zeros((n, max(1, g.model.mc_olen)), dtype=torch.float64, device="cuda")
    d_st = torch.zeros(n, dtype=torch.int32, device="cuda")
    d_it = torch.zeros(n, dtype=torch.int64, device="cuda")
    d_u = torch.zeros((g.ndof, S), dtype=torch.float64, device="cuda")
    vp = lambda x: (C.c_void_p * 1)(x.data_ptr())
    o = default_options()
    o.precision = precision
    o.tol = tol
    o.coarse = int(bool(coarse))
    _lib.check("ufem_mc_solve_device", L.ufem_mc_solve_device(
        1, (C.c_void_p * 1)(g.h.value), np.array([n], np.int64).ctypes.data_as(C.POINTER(C.c_long)), vp(d_in),
        vp(d_out), vp(d_st), vp(d_it), vp(d_g), vp(d_u), C.byref(o)))
    return d_u[:, :n].T.cpu().numpy(), d_st.cpu().numpy()


def gpu_von_mises(model, row, u):
    """von Mises at the stored points 1-19 from the GPU result pass on u."""
    from ufem_b200 import meshgen as mg
    from ufem_b200.api import GpuModel
    ms = mg.model_for_sample(model, row)
    gs = GpuModel(ms)
    gs.fill_K(0)
    gs.add_loads()
    gs.add_disps()
    gs.set_u(u)
    gs.fill_K(1)
    _, vm = gs.stresses(ms.eLen, False)
    gs.close()
    return vm.reshape(ms.eLen, 27)[:, :19]


def ours(a):
    import ctypes as C
    import numpy as np
    import torch
    import torch.distributed as dist
    from ufem_b200 import _lib
    from ufem_b200.api import GpuModel
    from ufem_b200.mc import default_options, mc_solve_serial
    from ufem_b200 import meshgen as mg
    from ufem_b200.warm import WarmStart
    from ufem_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    L = _lib.load()
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(v):
        return shard.max_over_ranks(v, device=dev)

    # ---- set-up (not timed): train the warm start -----------------------------
    m, train, ev = warm_setup(a, rank)
    g = GpuModel(m)
    cols, logs, scale_col = mg.warm_features(m)
    ws = WarmStart(g, cols, logs, scale_col, n_modes=64, n_hidden=256, n_snapshots=512,
                   epochs=a.epochs, batch=256, lr=2e-3, n_coarse=a.coarse_modes)
    t0 = time.perf_counter()
    tstats = ws.train(train, precision=a.precision)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    ws.set_guess_mode(a.guess)

    opt = default_options()
    opt.precision = a.precision
    opt.tol = 1e-8
    opt.coarse = 0 if a.no_coarse else 1
    n = ev.shape[0]
    olen = m.mc_olen
    d_in = torch.from_numpy(ev).to(dev)
    d_out = torch.zeros((n, olen), dtype=torch.float64, device=dev)
    d_st = torch.zeros(n, dtype=torch.int32, device=dev)
    d_it = torch.zeros(n, dtype=torch.int64, device=dev)
    wst = _lib.WarmStats()

    def step_device():
        _lib.check("ufem_warm_solve", L.ufem_warm_solve(ws.h, n, d_in.data_ptr(), d_out.data_ptr(), d_st.data_ptr(),
                                                         d_it.data_ptr(), C.byref(opt), C.byref(wst)))

    for _ in range(a.warmup):
        step_device()
    torch.cuda.synchronize()
    launches = 0
    pcg_ms = pcg_bytes = 0.0
    pcg_launches = 0
    fallbacks = 0
    with ClockSampler(os.path.join(tempfile.gettempdir(), f"ufem_clocks_{rank}.csv")) as clk:
        step_device()  # one more untimed step once the sampler runs
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        step_wall, step_pcg = [], []
        for _ in range(a.steps):
            t_step = time.perf_counter()
            step_device()
            step_wall.append(1000.0 * (time.perf_counter() - t_step))
            step_pcg.append(wst.pcg_ms)
            launches += wst.kernel_launches
            pcg_ms += wst.pcg_ms
            pcg_bytes += wst.pcg_bytes
            pcg_launches += wst.pcg_launches
            fallbacks += wst.fallbacks
        e1.record()
        torch.cuda.synchronize()
        barrier()
    ms_step = max_over_ranks(e0.elapsed_time(e1)) / a.steps
    solves_step = n * world
    value = solves_step / (ms_step / 1000.0)
    status = d_st.cpu().numpy()
    iters = d_it.cpu().numpy()
    out_warm = d_out.cpu().numpy().copy()
    warm_info = {f: getattr(wst, f) for f, _ in wst._fields_}
    mcs = _lib.McStats()
    L.ufem_mc_get_stats(C.byref(mcs))
    phases = {k: round(mcs.phase_wall_ms[i], 3) for i, k in enumerate(["init", "S", "U", "R", "C1", "C3"])}

    # ---- e2e: host (pinned) inputs -> device -> ufem_warm_solve -> host outputs
    h_in = torch.from_numpy(ev).pin_memory()
    h_out = torch.zeros((n, olen), dtype=torch.float64).pin_memory()
    h_st = torch.zeros(n, dtype=torch.int32).pin_memory()
    h_it = torch.zeros(n, dtype=torch.int64).pin_memory()
    barrier()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(a.steps):
        d_in.copy_(h_in, non_blocking=True)
        step_device()
        h_out.copy_(d_out, non_blocking=True)
        h_st.copy_(d_st, non_blocking=True)
        h_it.copy_(d_it, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / a.steps
    h2d = ev.nbytes
    d2h = h_out.numel() * 8 + h_st.numel() * 4 + h_it.numel() * 8
    e2e_ok = bool(np.array_equal(h_out.numpy(), out_warm))

    # ---- the same samples by the other forms: guess x precision x coarse ----
    dd = {"in": d_in, "out": d_out, "st": d_st, "it": d_it}
    forms = []
    if not a.no_other:
        combos = [(a.guess, 3, 1), (a.guess, 3, 0), (a.guess, 2, 1), (a.guess, 2, 0), (1, a.precision, 1),
                  (1, 2, 1), (2, a.precision, 1), (a.guess, 1, 0), (a.guess, 0, 0)]
        seen = {(a.guess, a.precision, opt.coarse)}
        for gm, pr, co in combos:
            if (gm, pr, co) in seen:
                continue
            seen.add((gm, pr, co))
            row, out_f = warm_run(L, ws, dd, gm, pr, co, 1 if pr in (0, 1) else a.steps)
            row["outputs_max_rel_diff_vs_headline"] = float(np.abs(out_f - out_warm).max() / np.abs(out_warm).max())
            forms.append(row)
        L.ufem_warm_set_guess_mode(ws.h, a.guess)

    # ---- the same samples without a guess (one batched launch) --------------
    one = np.array([n], np.int64).ctypes.data_as(C.POINTER(C.c_long))
    d_out2 = torch.zeros_like(d_out)
    d_st2 = torch.zeros_like(d_st)
    d_it2 = torch.zeros_like(d_it)

    def cold_run(precision, coarse):
        o = default_options()
        o.precision = precision
        o.tol = 1e-8
        o.coarse = coarse
        cold_args = (1, (C.c_void_p * 1)(g.h.value), one, _vp([d_in]), _vp([d_out2]), _vp([d_st2]), _vp([d_it2]),
                     (C.c_void_p * 1)(), (C.c_void_p * 1)(), C.byref(o))
        torch.cuda.synchronize()
        e0.record()
        _lib.check("ufem_mc_solve_device", L.ufem_mc_solve_device(*cold_args))
        e1.record()
        torch.cuda.synchronize()
        cold_ms = e0.elapsed_time(e1)
        it_cold = d_it2.cpu().numpy()
        out_cold = d_out2.cpu().numpy()
        # precision 4 needs a guess: the library runs a launch without one in precision 3
        return {"precision": PREC[3 if precision == 4 else precision], "coarse": bool(coarse),
                "value": n / (cold_ms / 1000.0),
                "unit": "solves/s", "iters_mean": float(it_cold.mean()), "iters_max": int(it_cold.max()),
                "all_converged": bool((d_st2.cpu().numpy() == 0).all()),
                "outputs_max_rel_diff_vs_warm": float(np.abs(out_cold - out_warm).max() / np.abs(out_cold).max())}

    cold = cold_run(a.precision, 0)
    cold["method"] = "PCG from zero, Jacobi preconditioner"
    cold_coarse = None
    if tstats["coarse_modes"] and opt.coarse:
        cold_coarse = cold_run(a.precision, 1)
        cold_coarse["method"] = f"PCG from zero, Jacobi + coarse correction on {tstats['coarse_modes']} POD modes"
    del d_out2, d_st2, d_it2

    result = None
    if rank == 0:
        # ---- the plain method on a subset of the same samples ----------------
        sub = ev[:a.plain_samples]
        mc_solve_serial(g, ev[-2:], tol=1e-8)  # warm-up: one-time set-up of the plain path
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        o_plain, st_plain, it_plain = mc_solve_serial(g, sub, tol=1e-8)
        torch.cuda.synchronize()
        plain_t = time.perf_counter() - t0
        plain = sub.shape[0] / plain_t
        plain_diff = float(np.abs(o_plain - out_warm[:sub.shape[0]]).max() / np.abs(o_plain).max())
        # ---- the headline method against the FP64 oracle ----------------------
        parity, cpu_matched = None, None
        procs = host_cores()
        if a.oracle_samples > 0 and not a.no_cpu:
            rows = ev[:a.oracle_samples]
            u_gpu, st_gpu = solve_u(L, g, ws, rows, a.guess, a.precision, opt.coarse)
            L.ufem_warm_set_guess_mode(ws.h, a.guess)
            tight, tight_wall = oracle_leg(m, rows, EPS_ORACLE, procs)
            eu = evm = eo = 0.0
            rows_d = [(int(r[2]), int(r[3]), int(r[0])) for r in m.mc_vars[m.mc_ilen:] if r[1] == mg.MONTE_VTYPE_RES_D]
            ndf = g.ndoffld(m.nLen)
            for s in range(rows.shape[0]):
                uo, vmo = tight[s][0], tight[s][1]
                eu = max(eu, float(np.abs(u_gpu[s] - uo).max() / np.abs(uo).max()))
                vm = gpu_von_mises(m, rows[s], u_gpu[s])
                evm = max(evm, float(np.abs(vm - vmo).max() / np.abs(vmo).max()))
                want = np.array([uo[ndf[node * 7 + d - 1] - 1] for node, d, _ in rows_d])
                got = out_warm[s, [p for _, _, p in rows_d]]
                eo = max(eo, float(np.abs(got - want).max() / np.abs(want).max()))
            parity = {"samples": int(rows.shape[0]), "method": "the headline's guess, precision and coarse space, "
                      "solved to true relative residual 1e-8",
                      "oracle": "oracle/ufem_oracle.c (the reference's assembly and femEqsCGwJ restated, pinned "
                                "bit-exact against the reference build), reference stopping rule FEM_ZERO/10000",
                      "u_rel_err_vs_oracle": eu, "vm_rel_err_vs_oracle": evm,
                      "outputs_rel_err_vs_oracle": eo, "all_converged": bool((st_gpu == 0).all()),
                      "vm_points": "the brick's stored result points 1-19 of every element (fem/fem_e009.c:825)",
                      "errors": "max over samples of max|x - x_oracle| / max|x_oracle|"}
            # the CPU leg at the GPU's tolerance: the oracle's Jacobi PCG to
            # relative residual 1e-8, one process per host core
            matched, wall = oracle_leg(m, rows, -1e-8, procs, want_fields=False)
            cpu_matched = {"value": rows.shape[0] / wall, "unit": "solves/s", "cores": procs, "kind": "port",
                           "iters_mean": float(np.mean([r[2] for r in matched])),
                           "sample": f"{rows.shape[0]} evaluation samples, oracle Jacobi PCG (femEqsCGwJ restated) "
                                     f"to relative residual 1e-8 with assembly, {procs} processes ({wall:.1f} s)",
                           "oracle_tight_wall_s": tight_wall}
        uneven = None if a.no_uneven else uneven_section(a, rank, dev)
        peak, peak_kind = measured_peaks()
        static = None if a.no_static else static_section(a, peak)
        achieved = pcg_bytes / (pcg_ms / 1000.0) / 1e9 if pcg_ms > 0 else 0.0
        # DRAM traffic per launch: the ncu-measured traffic / algorithmic ratio
        # of this kernel (profiles/, a smaller case of the same kernel) times
        # this run's algorithmic bytes per launch
        traffic = None
        pf = PROFILE.get(a.precision, ("none", ""))[0]
        tf = os.path.join(ROOT, "profiles", pf)
        if os.path.exists(tf) and pcg_launches > 0:
            for line in open(tf):
                if line.startswith("traffic_over_algorithmic:"):
                    traffic = float(line.split(":")[1]) * pcg_bytes / pcg_launches
        # ---- CPU baseline: the reference on a bounded sample ------------------
        cpu = None
        if os.path.exists(REF_LIB) and not a.no_cpu:
            with tempfile.TemporaryDirectory() as d:
                files = ref_files([m], [ev[:max(1, procs)]], d)
                nref, wall = run_reference_sample(files, procs, 1, d)
            cpu = {"value": nref / wall, "unit": "solves/s", "cores": procs, "kind": "reference",
                   "sample": f"{procs} processes x 1 evaluation sample via monte_solution, SSOR PCG to the "
                             f"reference's rule ({wall:.1f} s)",
                   "matched_tolerance": cpu_matched}
        s2 = tstats["sigma2"][:64]
        result = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "fp32 inner / fp64 refinement" if a.precision in (1, 3, 4) else "f64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD.format(c=a.coarse_modes), "samples_per_step": solves_step, "rel_res": 1e-8,
                       "ndof": g.ndof, "precision": PREC[a.precision], "guess": GUESS[a.guess],
                       "l2_flush": "not needed: every per-sample vector is 0.49 GB (FP32) / 0.98 GB (FP64) at "
                                   "8192 samples, >> 126 MB L2",
                       "parallelism": f"samples sharded over {world} GPU(s), no collective"},
            "all_converged": bool(np.isin(status, [0, 4]).all()),
            "warm_start": {"guess": GUESS[a.guess], "coarse_modes": tstats["coarse_modes"] if opt.coarse else 0,
                           "iters_mean": float(iters.mean()), "iters_max": int(iters.max()),
                           "cold_iters_mean": cold["iters_mean"],
                           "iterations_saved_frac": 1.0 - float(iters.mean()) / cold["iters_mean"],
                           "guess_rel_err_mean": warm_info["guess_err_mean"],
                           "guess_rel_err_max": warm_info["guess_err_max"],
                           "fallback_rate": fallbacks / max(1, n * a.steps), "cold_cap": warm_info["cold_cap"],
                           "ms_guess": warm_info["ms_guess"], "ms_solve": warm_info["ms_solve"],
                           "pcg_phase_wall_ms": phases, "true_residual_passes": mcs.true_residual_passes,
                           "train": {"samples": int(train.shape[0]), "seconds": train_s,
                                     "cold_iters_mean": tstats["cold_iters_mean"],
                                     "ms_solve": tstats["ms_solve"], "ms_basis": tstats["ms_basis"],
                                     "ms_mlp": tstats["ms_train"], "epochs": tstats["epochs"],
                                     "loss_first": tstats["loss_first"], "loss_last": tstats["loss_last"],
                                     "pod_energy_mode64_over_mode1": (s2[63] / s2[0]) if s2[0] else None}},
            "oracle_parity": parity,
            "other_forms": forms,
            "batched_without_guess": cold,
            "batched_coarse_without_guess": cold_coarse,
            "plain_fp64_one_at_a_time": {"value": plain, "unit": "solves/s", "samples_timed": int(sub.shape[0]),
                                         "iters_mean": float(it_plain.mean()),
                                         "outputs_max_rel_diff_vs_warm": plain_diff},
            "speedup_vs_plain": value / plain,
            "roofline": {"bound": "hbm",
                         "kernel": (KERNEL_SPLIT if a.precision == 4 and tstats["coarse_modes"] and opt.coarse
                                    else KERNEL[a.precision] + (" + coarse phases (tcgen05)"
                                                                if tstats["coarse_modes"] and opt.coarse else "")),
                         "achieved": achieved, "peak": peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "pcg_ms_per_step": pcg_ms / a.steps,
                         "pcg_launches_per_step": pcg_launches / a.steps},
            "e2e": {"value": solves_step / (e2e_ms / 1000.0), "unit": "solves/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "matches_device_run": e2e_ok},
            "gpu_launches": launches, "clocks": clk.summary(local),
            "step_wall_ms": [round(t, 1) for t in step_wall],
            "step_pcg_ms": [round(t, 1) for t in step_pcg],
            "uneven_batch": uneven,
            "static_configs": static,
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
        profile_case(a)
        return
    if a.profile_static:
        profile_static(a)
        return
    if a.profile_outputs:
        profile_outputs(a)
        return
    if a.profile_ingest:
        profile_ingest(a)
        return
    if a.impl == "reference":
        reference_arm(a)
    else:
        ours(a)


if __name__ == "__main__":
    main()
