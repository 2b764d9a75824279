"""Benchmark: SIMPLE iterations per second of the flow-solver pass on a B200,
learned initial guess + FP32-refined pressure solve against the plain FP64
path, both to the same 1e-8 pressure residual.

Workload (the headline metric's configuration): box of 2*128 x 128 x 128 =
4,194,304 hexahedral cells on a 0.2 x 0.1 x 0.1 m domain, inlet u = 50 m/s on
x-min, zero-gradient outlet on x-max, walls elsewhere, rho 1.2, mu 1.8e-5,
T0 1500 K; initial u, v, w, p, T = inlet state + seeded uniform noise +-1%;
1,000 seeded Gaussian particle-source blobs (momentum, energy, mass; sigma 2
cells, amplitude 1e-3 of the cell inflow); the corrected SIMPLE pass
(MC_MODE_SIMPLE), momentum URF 0.7, pressure URF 0.3, pressure PCG with the
aggregation-AMG V-cycle (or Jacobi, --psolver jacobi) to rtol 1e-8,
momentum/temperature BiCGStab to rtol 1e-8.  Synthetic data (the
reference has no dataset); the working set (about 4.5 GB) is far larger than
L2, so consecutive iterations stream from HBM.

One step = one SIMPLE pass (gradients, momentum assembly and three solves,
Rhie-Chow mass flux, pressure-correction assembly, PCG solve(s) and
corrections, temperature assembly and solve).

Two configurations run back to back from the same initial state:
  headline ("value"): MC_GUESS_LEARNED (the committed trained parameters) +
    MC_PRECISION_FP32_REFINED, pressure PCG-AMG;
  plain ("plain_fp64"): zero guess, FP64 PCG-AMG.
Field error: after the timed runs, each configuration runs --oracle-passes
untimed passes from the initial state and is compared with the CPU oracle
(oracle/liboracle.so, every solve to 1e-12, on the host's cores) after the
same passes: max relative difference per field.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs N independent replicas (the path is single-GPU: there is one
GPU's worth of work per replica and no data exchange between them), one per
rank under torchrun, and reports the whole-job rate.
"""
import argparse
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

from minicombust_app_b200 import replicas  # noqa: E402
from minicombust_app_b200.workload import (blob_phases, blob_stencils, gaussian_blobs, noisy_fields,  # noqa: E402
                                           varying_sources)

METRIC = "SIMPLE iters/s at 4.2M cells: learned+FP32-refined vs plain FP64, same 1e-8 residual"
UNIT = "iters/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--m", type=int, default=128, help="mesh modifier: 2m x m x m cells")
    ap.add_argument("--blobs", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-roofline", action="store_true")
    ap.add_argument("--psolver", default="amg", choices=["amg", "jacobi"],
                    help="pressure-correction preconditioner of the plain path (aggregation AMG or Jacobi)")
    ap.add_argument("--no-field-check", action="store_true", help="skip the comparison with the CPU oracle")
    ap.add_argument("--oracle-passes", type=int, default=3, help="passes compared with the CPU oracle")
    ap.add_argument("--source-period", type=int, default=0,
                    help="> 0: blob amplitudes vary as sin(2 pi pass / period + random phase), sources updated "
                         "on the device every pass (the largest benchmark configuration)")
    ap.add_argument("--reorder", default="none", choices=["none", "rcm"], help="cell order inside the solver")
    ap.add_argument("--amg-sweeps", type=int, default=None, help="override the V-cycle sweeps (both configurations)")
    ap.add_argument("--amg-cheb-ratio", type=float, default=None, help="override the Chebyshev ratio (both)")
    ap.add_argument("--ref-sample-m", type=int, default=48,
                    help="--impl reference: each step is one reference pass on the 2m x m x m box")
    ap.add_argument("--config", default="both", choices=["both", "headline", "plain"],
                    help="which configurations to time (default: both; value = headline)")
    return ap.parse_args()


# ------------------------------------------------------------------ inputs

# ------------------------------------------------------------------ clocks

class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=3.0):
        """Block until the sampler has produced a line, so that the samples
        cover the timed region from its start."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.01)

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() in ("active", "1"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------- roofline

def kernel_bytes(name, N, F, nnz_off):
    """Algorithmic (unique-touch) bytes of one launch: each stored input
    element read once, each output written once, at its stored type.  On a
    structured box the FP64 momentum and temperature rows and the FP32
    copies are stored by direction and the solver kernels read no column
    data (the assembly reads a 4-byte direction code per row).  The pressure
    solvers' FP64 copy is stored by direction in the half form of a
    symmetric matrix: the diagonal and the +x, +y, +z couplings, the others
    read as the neighbours' (counted once).  ELL values include the boundary
    padding."""
    return {
        "pcg_iter1_spmv": 64 * N,      # diag, 3 off, (z, p) pair -> p, q
        "pcg32_iter1_spmv": 44 * N,    # FP32: diag, 6 off by direction, (z, p) pair -> p, q
        "pcg_iter2_update": 64 * N,    # x rw, r rw, p, q, diag -> z (Jacobi path)
        "bicg3_1_spmv": 200 * N,       # matrix 56 + 3 x (r, p, v gathered; r0; p, v out)
        "bicg3_2_spmv": 152 * N,       # matrix 56 + 3 x (r, v gathered; s, t out)
        "bicg3_3_update": 168 * N,     # 3 x (s, p, t, r0, x rw, r out)
        "bicg3_32_1_spmv": 100 * N,    # FP32: matrix 28 + 3 x 24
        "bicg3_32_2_spmv": 76 * N,     # FP32: matrix 28 + 3 x 16
        "bicg3_32_3_update": 84 * N,
        "gnn_layers": 129 * N,         # one tcgen05 layer launch: h in 64, h out 64, mask 1 (four per pass)
        # one V-cycle, per fine row.  FP32 (every level's matrix by direction;
        # level 0's off-diagonal values read in FP16, 12 bytes), level 0:
        # first two sweeps 24, sweep 28, restriction 28, prolongation + sweep
        # 32, sweep 28, last sweep with r.z 28 = 168; level 1 (1/8 of the
        # rows, about 241 bytes per row) 30; level 2 and below 4
        "amg32_vcycle": 202 * N,
        # FP64 (level 0 in the half form: 32 bytes of matrix per row, coarse
        # levels by direction), level 0: first sweep 24, sweeps 4 x 56,
        # restriction 53, prolongation 21, last sweep 56 = 378; level 1 66;
        # level 2 and below 9
        "amg_vcycle": 453 * N,
        "lsq_gradients_uvwpt": 208 * N,
        # a cell's faces: face index, other cell (col) and owner bits per
        # cell instead of each face's two cell indices
        "momentum_assemble": 48 * F + 325 * N,
        "mass_flux": 88 * F + 176 * N,
        # faces: mdot, ff0, ff1; cells: face index, other cell, owner bits,
        # code -> b, diag, six values, the FP64 copy in the half form (the
        # FP32 level 0 the refined configuration also writes, 28 N, is not
        # counted)
        "pressure_rows": 24 * F + 141 * N,
        "temperature_assemble": 40 * F + 172 * N,
    }.get(name)


# DRAM bytes per row (read + write) of one launch, measured with ncu on the
# 2 x 96^3 case (a full capture of the 2 x 128^3 case is too large); scaled by
# rows to the bench size for the roofline's `traffic`.
NCU_DRAM_BYTES_PER_ROW = {
    "bicg3_1_spmv": 217.2,   # k_bicg_1<double,3>: 384.3 MB read + written on 1,769,472 cells
    "gnn_layers": 103.6,     # k_gnn_layer_umma: 115.1 + 68.2 MB read + written on 1,769,472 cells
}

# Timed groups that are several kernel launches: the four layer launches of
# the network are timed as one group.
KERNELS_PER_GROUP = {"gnn_layers": 4}
# Timed groups made of different kernels (one V-cycle: 25 kernels in FP32, 21
# in FP64 on the benchmark box); they get per-group figures but are not the
# line's roofline kernel, which is one kernel.
COMPOSITE = ("amg_vcycle", "amg32_vcycle")


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------- reference arm

def host_threads():
    """Host threads for the CPU checkers: all but two of the cores this
    process may use (one drives the GPU)."""
    try:
        n = len(os.sched_getaffinity(0))
    except Exception:
        n = os.cpu_count() or 1
    return max(1, n - 2)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


def seeded_reference(m):
    """The reference's own CPU FlowSolver (oracle/_ref, its physics) on the
    2m x m x m box, seeded like the benchmark, solves to 1e-8."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import Reference, noisy_initial_fields
    ref = Reference(2 * m, m, m, 0.2, 0.1, 0.1, delta=1.0e-5, bcgs_rtol=1e-8, cg_rtol=1e-8)
    init = noisy_initial_fields(ref.N, {"U": 50.0, "V": 0.0, "W": 0.0, "P": 4000.0, "TEM": 2000.0}, 0)
    for name, vals in init.items():
        a = ref.field(name)
        a[:ref.N] = vals
        ref.set_field(name, a)
    return ref


def run_reference_arm(args, rank, world):
    """Each step is one real SIMPLE pass of the reference on the sample box
    (the reference's flow loops are serial: one core); the metric scales the
    measured per-cell rate to the benchmark box.  Warm-up: one pass."""
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import ref_available
    if not ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmcref.so (the reference compiled "
                                                              "from its sources) is not built"}))
        return
    sm = args.ref_sample_m
    ref = seeded_reference(sm)
    ref.step()  # warm-up; the first pass also runs set_up_field
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.step()
        times.append(time.perf_counter() - t0)
    ref.close()
    per_pass = float(np.mean(times))
    scale = (2 * args.m ** 3) / (2 * sm ** 3)
    value = 1.0 / (per_pass * scale)
    sample = (f"{args.steps} real SIMPLE passes of the reference CPU FlowSolver (its own physics, solves to 1e-8, "
              f"1 core of {cpu_model()}) on 2*{sm}^3 = {2 * sm ** 3} cells after 1 warm-up pass; {per_pass:.2f} s "
              f"per pass, rate scaled by cell count x {scale:.1f} to 2*{args.m}^3")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * per_pass, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"reference CPU FlowSolver, box 2*{args.m}^3 cells (one step = one pass on the "
                                   f"2*{sm}^3 sample box)", "cells": 2 * args.m ** 3, "sample_cells": 2 * sm ** 3,
                       "mode": "reference physics", "warmup_passes_run": 1},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": 1, "kind": "reference", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def oracle_run(m, blobs, passes, rtol, threads, warm=0, period=0):
    """The CPU oracle (the C restatement, simple mode) on the benchmark box
    from the benchmark's initial state: fields after warm + passes passes,
    and the seconds per pass of the last `passes` (with period > 0 the
    time-varying sources of each pass are set before it)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from checkers import SIMPLE, Oracle, oracle_lib, oracle_mesh, oracle_params
    dims, lengths = (2 * m, m, m), (0.2, 0.1, 0.1)
    oracle_lib().mco_set_threads(threads)
    orc = Oracle(oracle_mesh(*dims, *lengths), oracle_params(SIMPLE, u_rtol=rtol, p_rtol=rtol))
    for name, vals in noisy_fields(orc.N, seed=0).items():
        a = orc.field(name)
        a[:orc.N] = vals
        orc.set_field(name, a)
    if period > 0:
        stencils, phases = blob_stencils(dims, lengths, blobs, seed=0), blob_phases(blobs, seed=0)
    else:
        orc.set_sources(gaussian_blobs(dims, lengths, blobs, seed=0))
    it = 0
    for _ in range(warm):
        if period > 0:
            orc.set_sources(varying_sources(orc.N, stencils, phases, it, period))
        if orc.step() != 0:
            raise RuntimeError("oracle solve did not converge")
        it += 1
    t0 = time.perf_counter()
    for _ in range(passes):
        if period > 0:
            orc.set_sources(varying_sources(orc.N, stencils, phases, it, period))
        if orc.step() != 0:
            raise RuntimeError("oracle solve did not converge")
        it += 1
    dt = (time.perf_counter() - t0) / passes
    fields = {n: orc.field(n)[:orc.N].copy() for n in FIELD_NAMES}
    orc.close()
    return fields, dt


# ------------------------------------------------------------------- main

FIELD_NAMES = ("U", "V", "W", "P", "TEM")


def make_solver(flow, mesh, dims, lengths, args, rank, local, headline):
    """The benchmark solver of one configuration, seeded identically."""
    reorder = flow.REORDER_RCM if args.reorder == "rcm" else flow.REORDER_NONE
    if headline:
        from minicombust_app_b200 import train_guess
        params = flow.default_params(flow.MODE_SIMPLE, device=local, p_rtol=1e-8, u_rtol=1e-8,
                                     pressure_solver=flow.PSOLVER_PCG_AMG, precision=flow.PRECISION_FP32_REFINED,
                                     initial_guess=flow.GUESS_LEARNED, reorder=reorder)
    else:
        psolver = flow.PSOLVER_PCG_AMG if args.psolver == "amg" else flow.PSOLVER_PCG_JACOBI
        params = flow.default_params(flow.MODE_SIMPLE, device=local, p_rtol=1e-8, u_rtol=1e-8,
                                     pressure_solver=psolver, reorder=reorder)
    if args.amg_sweeps is not None:
        params.amg_sweeps = args.amg_sweeps
    if args.amg_cheb_ratio is not None:
        params.amg_cheb_ratio = args.amg_cheb_ratio
    solver = flow.FlowSolver(mesh, params=params)
    if headline:
        solver.set_guess_params(train_guess.load_params())
    N = solver.N
    for name, vals in noisy_fields(N, seed=rank).items():
        a = solver.field(name)
        a[:N] = vals
        solver.set_field(name, a)
    if args.source_period <= 0:
        solver.set_sources(gaussian_blobs(dims, lengths, args.blobs, seed=rank))
    return solver


class VaryingSources:
    """The time-varying blob sources on the device: g = G w(pass), G the
    [cells x blobs] stencil matrix (CSR), w_b = sin(2 pi pass / period +
    phase_b); sources [5][cells] = (g, 0, 0, 1e3 g, 1e-2 g), handed to the
    solver with mc_flow_set_sources_device on its stream every pass."""

    def __init__(self, torch, dims, lengths, blobs, period, seed, device):
        cells, values, blob = blob_stencils(dims, lengths, blobs, seed)
        n = dims[0] * dims[1] * dims[2]
        G = torch.sparse_coo_tensor(np.stack([cells, blob]), values, (n, blobs), dtype=torch.float64)
        self.G = G.coalesce().to_sparse_csr().to(device)
        self.phases = torch.tensor(blob_phases(blobs, seed), dtype=torch.float64, device=device)
        self.coef = torch.tensor([1.0, 0.0, 0.0, 1.0e3, 1.0e-2], dtype=torch.float64, device=device)
        self.src = torch.zeros((5, n), dtype=torch.float64, device=device)
        self.period = period
        self.torch = torch

    def apply(self, solver, stream, it):
        torch = self.torch
        with torch.cuda.stream(stream):
            w = torch.sin(2.0 * np.pi * it / self.period + self.phases)
            g = (self.G @ w.unsqueeze(1)).squeeze(1)
            torch.outer(self.coef, g, out=self.src)
        solver.set_sources_device(self.src.data_ptr())


def timed_steps(torch, solver, stream, steps, barrier, max_over_ranks, local, sources=None, it0=0):
    """Device-timed SIMPLE passes (CUDA events on the solver's stream,
    barrier + synchronize on both sides, max over ranks), clocks sampled;
    with time-varying sources each pass first updates them on the device."""
    stats = []
    launches0 = solver.launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_first()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for k in range(steps):
        if sources is not None:
            sources.apply(solver, stream, it0 + k)
        solver.simple_iteration()
        stats.append(solver.last_stats.as_dict())
    ev1.record(stream)
    barrier()
    clocks = sampler.stop()
    t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    return t, stats, clocks, solver.launch_count() - launches0


def working_launches(name, st, launches):
    """Launches of a kernel in the instrumented pass that did work: the
    host-polled batches of that pass also launch iterations that find their
    solve converged and return at once.  One V-cycle and one product per
    PCG iteration, one BiCGStab triple per iteration; assembly kernels run
    once per pass."""
    it = None
    if name in KERNELS_PER_GROUP:
        return launches * KERNELS_PER_GROUP[name]
    if name in ("amg32_vcycle", "amg_vcycle", "pcg_iter1_spmv", "pcg32_iter1_spmv"):
        it = st["pressure_iters_total"]
    elif name.startswith("bicg3"):
        it = max(st["momentum_iters"])
    elif name.startswith("bicg1"):
        it = st["temperature_iters"]
    if it is None or it <= 0 or it > launches:
        return launches
    return it


def roofline_of(solver, mesh, N):
    """One instrumented pass: for every kernel with a byte model, its
    CUDA-event time, launches (all, and those that did work) and achieved
    bandwidth; the single kernel with the largest time is the line's
    roofline (a V-cycle, a group of different kernels, is listed but not
    chosen)."""
    solver.reset_kernel_times()
    solver.set_timing(True)
    solver.simple_iteration()
    solver.set_timing(False)
    kt = solver.kernel_times()
    st = solver.last_stats.as_dict()
    nnz_off = int(np.sum(mesh.face_cells[:, 1] < N)) * 2
    total = sum(v[0] for v in kt.values())
    peak, kind = measured_peaks()
    per_kernel = {}
    for name, (ms, cnt) in kt.items():
        b = kernel_bytes(name, N, mesh.n_faces, nnz_off)
        if cnt == 0 or b is None:
            continue
        work = working_launches(name, st, cnt)
        avg_s = ms / work / 1e3
        launches = cnt * KERNELS_PER_GROUP.get(name, 1)
        per_kernel[name] = {"ms": round(ms, 4), "launches": launches, "working_launches": work,
                            "bytes_per_launch": b, "avg_launch_us": round(avg_s * 1e6, 2),
                            "achieved_gbs": round(b / avg_s / 1e9, 1), "frac": round(b / avg_s / 1e9 / peak, 3),
                            "share_of_step": round(ms / total, 4)}
    roof = None
    single = [k for k in per_kernel if k not in COMPOSITE]
    if single:
        name = max(single, key=lambda k: per_kernel[k]["ms"])
        k = per_kernel[name]
        row = NCU_DRAM_BYTES_PER_ROW.get(name)
        roof = {"kernel": name, "bound": "hbm", "achieved": k["achieved_gbs"], "peak": peak, "unit": "GB/s",
                "frac": k["frac"], "peak_source": kind,
                "traffic": row * N if row else None,
                "traffic_source": "ncu dram__bytes_read+write on 2x96^3, scaled by rows" if row else None,
                "bytes_per_launch": k["bytes_per_launch"], "avg_launch_us": k["avg_launch_us"],
                "launches_per_step": k["working_launches"],
                "early_exit_launches": k["launches"] - k["working_launches"], "share_of_step": k["share_of_step"]}
    return roof, {k: round(v[0], 4) for k, v in kt.items() if v[1] > 0}, per_kernel


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as tdist
        from datetime import timedelta
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=timedelta(seconds=600))
        dist = tdist
    torch.cuda.set_device(local)

    from minicombust_app_b200 import build as mcbuild
    from minicombust_app_b200 import flow
    if not os.path.exists(flow.LIB_PATH):
        mcbuild.build()

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return replicas.max_over_ranks(x, dist, device="cuda")

    m = args.m
    dims, lengths = (2 * m, m, m), (0.2, 0.1, 0.1)
    mesh = flow.Mesh.box(*dims, *lengths)
    N = mesh.n_cells
    sources = None
    if args.source_period > 0:
        sources = VaryingSources(torch, dims, lengths, args.blobs, args.source_period, rank,
                                 torch.device("cuda", local))
    runs = {}
    order = {"both": ("plain", "headline"), "headline": ("headline",), "plain": ("plain",)}[args.config]
    for cfg in order:
        solver = make_solver(flow, mesh, dims, lengths, args, rank, local, cfg == "headline")
        stream = torch.cuda.ExternalStream(solver.stream(), device=torch.device("cuda", local))
        for k in range(args.warmup):
            if sources is not None:
                sources.apply(solver, stream, k)
            solver.simple_iteration()
        t, stats, clocks, launches = timed_steps(torch, solver, stream, args.steps, barrier, max_over_ranks, local,
                                                 sources, args.warmup)
        fields = {n: solver.field(n)[:N].copy() for n in FIELD_NAMES} if rank == 0 else None
        r = {"t": t, "stats": stats, "clocks": clocks, "launches": launches, "fields": fields}
        if cfg == order[-1]:
            # end to end through the C ABI with pinned host buffers: every
            # step uploads the five fields and reads them back
            pinned = {n: torch.empty(N + 6, dtype=torch.float64, pin_memory=True) for n in FIELD_NAMES}
            for n in FIELD_NAMES:
                pinned[n].numpy()[:] = solver.field(n)
            L, h = flow.library(), solver.h
            barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for k in range(args.steps):
                for n in FIELD_NAMES:
                    flow._check(L.mc_flow_set_field(h, flow.FIELDS[n], pinned[n].data_ptr()), h, "set_field")
                if sources is not None:
                    sources.apply(solver, stream, args.warmup + args.steps + k)
                solver.simple_iteration()
                for n in FIELD_NAMES:
                    flow._check(L.mc_flow_get_field(h, flow.FIELDS[n], pinned[n].data_ptr()), h, "get_field")
            e1.record(stream)
            barrier()
            r["e2e"] = replicas.whole_job_rate(args.steps, max_over_ranks(e0.elapsed_time(e1) / 1e3), world)
            r["e2e_bytes"] = 5 * (N + 6) * 8
        if rank == 0 and not args.no_roofline:
            r["roofline"], r["kernel_ms"], r["kernels"] = roofline_of(solver, mesh, N)
        runs[cfg] = r
        solver.close()

    # field error against the CPU oracle: each configuration re-runs
    # oracle_passes untimed passes from the initial state
    oracle_cmp = None
    if rank == 0 and not args.no_field_check and args.oracle_passes > 0:
        P = args.oracle_passes
        gpu_fields = {}
        for cfg in order:
            sv = make_solver(flow, mesh, dims, lengths, args, rank, local, cfg == "headline")
            sv_stream = torch.cuda.ExternalStream(sv.stream(), device=torch.device("cuda", local))
            for k in range(P):
                if sources is not None:
                    sources.apply(sv, sv_stream, k)
                sv.simple_iteration()
            gpu_fields[cfg] = {n: sv.field(n)[:N].copy() for n in FIELD_NAMES}
            sv.close()
        threads = host_threads()
        ofields, _ = oracle_run(m, args.blobs, P, 1e-12, threads, period=args.source_period)
        oracle_cmp = {"passes": P, "oracle": "CPU oracle (C restatement), simple mode, solves to 1e-12",
                      "oracle_threads": threads}
        for cfg in order:
            oracle_cmp[cfg] = {n: float(np.abs(gpu_fields[cfg][n] - ofields[n]).max()
                                        / max(np.abs(ofields[n]).max(), 1e-300)) for n in FIELD_NAMES}

    if rank == 0:
        main_cfg = order[-1]
        R = runs[main_cfg]
        value = replicas.whole_job_rate(args.steps, R["t"], world)
        cpu = None
        if not args.no_cpu_baseline:
            # a real pass of the CPU oracle (the port) on the benchmark box at
            # the benchmark's tolerances, on the host's cores
            threads = host_threads()
            _, per_pass = oracle_run(m, args.blobs, 1, 1e-8, threads, warm=1, period=args.source_period)
            cpu = {"value": 1.0 / per_pass, "unit": UNIT, "cores": threads, "kind": "port",
                   "sample": f"1 real SIMPLE pass of the CPU oracle (C restatement, simple mode, solves to 1e-8, "
                             f"unpreconditioned CG for the pressure correction) on the full 2*{m}^3 box after its "
                             f"first pass, {threads} threads of {cpu_model()}: {per_pass:.1f} s"}
        summary = {}
        for cfg, r in runs.items():
            pit = [st["pressure_iters_total"] for st in r["stats"]]
            summary[cfg] = {"value": replicas.whole_job_rate(args.steps, r["t"], world),
                            "ms_per_step": 1e3 * r["t"] / args.steps,
                            "pressure_iters_per_step": float(np.mean(pit)),
                            "guess_rel_residual": float(np.mean([st["guess_rel_residual_first"] for st in r["stats"]])),
                            "momentum_iters": r["stats"][-1]["momentum_iters"],
                            "temperature_iters": r["stats"][-1]["temperature_iters"],
                            "pressure_rel_residual": max(st["pressure_rel_residual"] for st in r["stats"]),
                            "mass_imbalance": r["stats"][-1]["mass_imbalance"], "gpu_launches": r["launches"],
                            "pressure_rel_residual_first": float(np.mean([st["pressure_rel_residual_first"]
                                                                          for st in r["stats"]])),
                            "roofline": r.get("roofline"), "kernel_ms_one_step": r.get("kernel_ms"),
                            "kernels": r.get("kernels")}
        desc = ("learned initial guess + FP32-refined pressure PCG-AMG (FP64 outer refinement)"
                if main_cfg == "headline" else "plain FP64 path, pressure PCG-AMG")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * R["t"] / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if main_cfg == "headline" else "f64",
                "data": "synthetic",
                "config": {"workload": f"simple-mode SIMPLE pass, box 2*{m}x{m}x{m} = {N} cells, {args.blobs} "
                                       + ("source blobs, " if args.source_period <= 0 else
                                          f"source blobs with amplitudes sin(2 pi pass / {args.source_period} + "
                                          "random phase) updated on the device every pass, ")
                                       + f"{desc}, BiCGStab momentum/T, rtol 1e-8"
                                       + (", RCM cell order" if args.reorder == "rcm" else ""),
                           "cells": N, "faces": mesh.n_faces, "l2": "inputs larger than L2 (~4.5 GB working set)",
                           "parallelism": "replicas" if world > 1 else "single GPU"},
                "e2e": {"value": R["e2e"], "unit": UNIT, "h2d_bytes_per_step": R["e2e_bytes"],
                        "d2h_bytes_per_step": R["e2e_bytes"]},
                "gpu_launches": R["launches"], "clocks": R["clocks"], "roofline": R.get("roofline"),
                "cpu_baseline": cpu, "configs": summary,
                "field_rel_error_vs_fp64_oracle": oracle_cmp}
        if "plain" in runs and "headline" in runs:
            line["speedup_vs_plain_fp64"] = summary["headline"]["value"] / summary["plain"]["value"]
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
