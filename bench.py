"""Benchmark of the neo-Hookean hot path on B200.

Workload: the 64^3-cube five-tet box (274,625 vertices, 1,310,720 tets, 3,494,465 3x3
blocks) with per-element mu log-uniform in [1e3, 1e5], nu ~ U[0.30, 0.45], bottom face
fixed, gravity -9.8 z, density 1000 (seeded synthetic data).

One step = one FP64 evaluation of energy + gradient + exact block-CSR Hessian of the whole
mesh. `value` is tets/s over K device-timed steps with inputs resident in HBM; `e2e` is the
same metric through the C ABI (lpg_fem_eval) with pinned HOST buffers, i.e. including the
H2D copy of u and the D2H copy of the gradient and the Hessian (reference CSC order) every
step. The Newton time-to-1e-8 (relative gradient norm, Armijo backtracking) of the mixed
FP32/FP64 path and of the FP64 path is reported beside it.

  python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--no-newton]
"""

import argparse
import ctypes
import json
import os
import platform
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "neo-Hookean tets/s (E+∇+BSR Hessian); Newton time-to-1e-8, mixed vs FP64"
N_CUBES = 64


def workload_config():
    from litepgo_b200 import mesh

    V, T, nnzb = mesh.box_counts(N_CUBES)
    return {
        "workload": f"gravity box {N_CUBES}^3 cubes x 5 tets (V={V}, T={T}, nnzb={nnzb}), per-element mu "
                    "log-uniform [1e3,1e5], nu U[0.30,0.45], z=0 fixed, gravity -9.8, rho 1000, seed 0",
        "step": "one FP64 E + gradient + exact 3x3 block-CSR Hessian evaluation of the whole mesh",
        "state": "u = (A - I) X + 1e-3 N(0,1), A = I + 0.1 N(0,1) (seed 11)",
        "l2": "working set per step ~412 MB (element records 126 MB, Hessian 252 MB) > 126 MB L2",
        "tets": T, "vertices": V, "nnzb": nnzb,
    }


def state(X):
    rng = np.random.default_rng(11)
    A = np.eye(3) + 0.1 * rng.standard_normal((3, 3))
    return (X @ A.T - X + 0.001 * rng.standard_normal(X.shape)).ravel()


def algorithmic_bytes(T, V, nnzb, precision="f64"):
    """Compulsory traffic of one E+grad+H evaluation: per tet indices, record (G, vol, theta),
    per vertex u in and gradient out, 9 values per block out."""
    if precision == "f64":
        return T * (16 + 72 + 8 + 16) + V * (24 + 24) + 72 * nnzb
    return T * (16 + 36 + 4 + 8) + V * (12 + 12) + 36 * nnzb


class ClockSampler:
    """SM clock and clock-event reasons sampled every 2 ms during the timed region.

    Reads NVML in a background thread (read-only queries; the device is matched to the CUDA
    device by PCI bus id); falls back to nvidia-smi at its 200 ms cadence without NVML.
    """

    REASONS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
               "sw_power_cap": 0x4}

    def __init__(self, cuda_device):
        self.cuda_device = cuda_device
        self.samples = []  # (sm_mhz, reasons bitmask)
        self.max_mhz = None
        self.stop = threading.Event()
        self.thread = None
        self.proc = None
        self.lines = []

    def _handle(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        props = torch.cuda.get_device_properties(self.cuda_device)
        try:
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.cuda_device)

    def _poll(self, nv, h):
        reasons_fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
            nv.nvmlDeviceGetCurrentClocksThrottleReasons
        while not self.stop.is_set():
            try:
                self.samples.append((nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM), int(reasons_fn(h))))
            except Exception:
                pass
            time.sleep(0.002)

    def __enter__(self):
        try:
            nv, h = self._handle()
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll, args=(nv, h), daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
            try:
                fields = "clocks.sm,clocks.max.sm,clocks_event_reasons.active"
                self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                                              "-i", str(self.cuda_device), "-lms", "200"], stdout=subprocess.PIPE,
                                             stderr=subprocess.DEVNULL, text=True)
                threading.Thread(target=lambda: self.lines.extend(l.strip() for l in self.proc.stdout),
                                 daemon=True).start()
            except (FileNotFoundError, OSError):
                self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            time.sleep(0.004)
            self.stop.set()
            self.thread.join(timeout=2)
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            try:
                self.samples.append((float(parts[0]), int(parts[2], 16)))
                self.max_mhz = float(parts[1])
            except (ValueError, IndexError):
                continue

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": [], "samples": 0}
        reasons = sorted(n for n, bit in self.REASONS.items() if any(r & bit for _, r in self.samples))
        return {"sm_mhz": statistics.median(s for s, _ in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples)}


def profile_traffic():
    """Per-launch DRAM bytes of the assembly kernel from the committed ncu summary, if any."""
    p = ROOT / "profiles" / "tet_cluster_kernel_f64_exact_64cube.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except (KeyError, ValueError):
            pass
    return 6650.0, "fallback"


def cpu_model():
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def _median_eval_seconds(m, u, runs=5, warm=2):
    """The reference benchmark's method (benchmarks/torch_material.py:50-59, 207-219): one cold
    call, `warm` warm-up calls, then the median of `runs` timed calls of E + gradient + exact
    CSC Hessian."""
    m.eval(u, True, 1)
    for _ in range(warm):
        m.eval(u, True, 1)
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        m.eval(u, True, 1)
        times.append(time.perf_counter() - t0)
    return float(np.median(times))


def cpu_baseline(X, tets, theta, u_full):
    """The oracle (the reference's CPU algorithm restated in C++/OpenMP) on the host cores: E +
    gradient + exact CSC Hessian, median of 5 after a cold call and 2 warm-ups, on the full mesh
    with every host thread, and with one thread on a slab of the mesh (its first eighth of cube
    layers, the same elements' evaluation per tet)."""
    import oracle

    oracle.set_threads(0)
    threads = oracle.get_threads()
    T = tets.shape[0]
    m = oracle.OracleMesh(X, tets, theta)
    med = _median_eval_seconds(m, u_full)
    del m
    # One thread on a slab: elements [0, T/8) of the cube-ordered box and their vertices.
    Ts = max(T // 8, 1)
    sub = tets[:Ts]
    verts, local = np.unique(sub, return_inverse=True)
    ms = oracle.OracleMesh(X[verts], local.reshape(-1, 4).astype(np.int32), theta[:Ts] if theta.ndim == 2 else theta)
    oracle.set_threads(1)
    med1 = _median_eval_seconds(ms, u_full.reshape(-1, 3)[verts].ravel())
    oracle.set_threads(0)
    return {"value": T / med, "unit": "tets/s", "cores": threads, "kind": "port",
            "sample": f"E+grad+exact CSC Hessian of the {T}-tet mesh: 1 cold call, 2 warm-ups, median of 5 "
                      f"({med:.3f} s) with {threads} OpenMP threads",
            "one_thread": {"value": Ts / med1, "unit": "tets/s", "cores": 1,
                           "sample": f"the same on the first {Ts} tets (their {verts.size} vertices), median of 5 "
                                     f"({med1:.3f} s) on one thread"},
            "cpu_model": cpu_model()}


def dist_setup(n_gpus):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def tuning_summary(fem_energy):
    """The launch variants the handle's autotuner chose, with its timings (ms; null = not timed)."""
    t = fem_energy.tuning()
    return {"choice": t["choice"],
            "ms": {k: [None if v != v else round(v, 4) for v in vals] for k, vals in t["ms"].items()}}


def whole_job_rate(units_per_rank, seconds_max, world):
    """Whole-job throughput of `world` identical replicas: all ranks' units over the slowest
    rank's time (the max over ranks)."""
    return world * units_per_rank / seconds_max


def run_reference(args):
    rank, world, _ = dist_setup(args.gpus)
    if rank != 0:
        return 0
    from litepgo_b200 import workloads

    g = workloads.gravity_box(N_CUBES, seed=0)
    u = state(g["X"])
    import oracle

    oracle.set_threads(0)
    threads = oracle.get_threads()
    m = oracle.OracleMesh(g["X"], g["tets"], g["theta"])
    T = g["tets"].shape[0]
    m.eval(u, True, 1)  # cold call
    for _ in range(max(args.warmup, 0)):
        m.eval(u, True, 1)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        m.eval(u, True, 1)
        times.append(time.perf_counter() - t0)
    el = float(np.sum(times))
    med = float(np.median(times))
    value = T / med
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "tets/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": workload_config(),
        "cpu_baseline": {"value": value, "unit": "tets/s", "cores": threads, "kind": "port",
                         "sample": f"median of {args.steps} full evaluations (E+grad+exact CSC Hessian) of the {T}-tet "
                                   f"mesh after a cold call and {args.warmup} warm-ups, by the C++/OpenMP restatement "
                                   f"of the reference CPU path, {threads} threads",
                         "cpu_model": cpu_model()},
        "e2e": {"value": value, "unit": "tets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference itself cannot be built here (Eigen 5 / oneTBB / nanobind fetched at configure time, "
                "no network); this arm times its algorithm restated in oracle/",
    }
    print(json.dumps(line), flush=True)
    return 0


def newton_times(fem_energy, g, torch):
    """Newton to a 1e-8 relative gradient norm with Armijo backtracking: mixed vs FP64."""
    from litepgo_b200 import dof, energy, solver

    import scipy.sparse as sp

    n = g["X"].size
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"])
    total = energy.WeightedSumEnergy([(fem_energy, 1.0), (load, 1.0)])
    fixed = dof.DofReduction(n, g["fixed"])
    out = {}
    x0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    for prec in ("mixed", "f64"):
        opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                    precision=prec, max_iterations=100, cg_tolerance=1e-2, cg_max_iterations=20000)
        # Untimed warm-up solve (2 Newton iterations): buffers of this precision and its PCG
        # graph exist before the timed solve, as in a solver called repeatedly.
        warm = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                    precision=prec, max_iterations=2, cg_tolerance=1e-2, cg_max_iterations=20000)
        solver.newton_solve(total, fixed, x0, warm)
        t0 = time.perf_counter()
        r = solver.newton_solve(total, fixed, x0, opts)
        wall = time.perf_counter() - t0
        out[prec] = {"status": r.status.name, "seconds": r.seconds, "wall_seconds": wall, "iterations": r.iterations,
                     "cg_iterations": int(r.cg_iterations), "relative_gradient": r.gradient_norm / max(r.gradient_norm0, 1e-300),
                     "line_search_evaluations": r.line_search_evaluations}
        out[prec + "_x"] = r.x
    xm, xf = out.pop("mixed_x"), out.pop("f64_x")
    out["max_abs_diff_mixed_vs_f64"] = float((xm - xf).abs().max().item())
    if out["mixed"]["seconds"] > 0:
        out["speedup_mixed_vs_f64"] = out["f64"]["seconds"] / out["mixed"]["seconds"]
    return out


def run_ours(args):
    import torch

    rank, world, local = dist_setup(args.gpus)
    from litepgo_b200 import _native as N
    from litepgo_b200 import energy, fem, workloads

    g = workloads.gravity_box(N_CUBES, seed=0)
    X, tets, theta = g["X"], g["tets"], g["theta"]
    T, V = tets.shape[0], X.shape[0]
    u_host = state(X)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta)
    dev = torch.device("cuda", torch.cuda.current_device())
    u = torch.as_tensor(u_host, device=dev)
    grad = torch.empty(3 * V, dtype=torch.float64, device=dev)
    hess = torch.empty(e.nnz, dtype=torch.float64, device=dev)
    Exact = energy.HessianKind.Exact

    def step():
        return e.eval_device(u, gradient=True, hessian=Exact, grad_out=grad, hess_out=hess)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local if world > 1 else torch.cuda.current_device()) as clocks:
        barrier(world)
        torch.cuda.synchronize()
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, world)
    ms_per_step = ms / args.steps
    value = whole_job_rate(T * args.steps, ms * 1e-3, world)
    gpu_launches = 3 * args.steps  # per step: the assembly kernel and the two-stage energy sum

    # Roofline of the assembly kernel: CUDA events on its launching stream, L2 flushed between launches.
    ma, me = ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_set_stream(e.handle, ctypes.c_void_p(stream.cuda_stream)))
    N.check(N.lib.lpg_fem_time_eval(e.handle, N.vptr(u), N.vptr(grad), int(Exact), N.PRECISION_F64, N.LAYOUT_BSR,
                                    N.vptr(hess), 10, 1, ctypes.byref(ma), ctypes.byref(me)))
    ab = algorithmic_bytes(T, V, e.nnzb, "f64")
    peak, peak_kind = measured_peak()
    achieved = ab / (ma.value * 1e-3) / 1e9
    traffic = profile_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "tet_cluster_kernel<double, gradient, exact Hessian>", "kernel_ms": ma.value,
                "algorithmic_bytes": ab, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    # Mixed (FP32 element arithmetic + FP32 Hessian) kernel, reported beside it.
    hess32 = torch.empty(e.nnz, dtype=torch.float32, device=dev)
    ma32, me32 = ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_time_eval(e.handle, N.vptr(u), N.vptr(grad), int(Exact), N.PRECISION_MIXED, N.LAYOUT_BSR,
                                    N.vptr(hess32), 10, 1, ctypes.byref(ma32), ctypes.byref(me32)))
    ab32 = algorithmic_bytes(T, V, e.nnzb, "f32")
    mixed = {"tets_per_s_kernel": T / (ma32.value * 1e-3), "kernel_ms": ma32.value,
             "achieved_gbs": ab32 / (ma32.value * 1e-3) / 1e9, "frac": ab32 / (ma32.value * 1e-3) / 1e9 / peak,
             "algorithmic_bytes": ab32}

    # End to end through the C ABI with pinned host buffers (H2D of u, D2H of gradient + CSC Hessian).
    u_pin = torch.as_tensor(u_host).pin_memory()
    g_pin = torch.empty(3 * V, dtype=torch.float64).pin_memory()
    h_pin = torch.empty(e.nnz, dtype=torch.float64).pin_memory()
    N.check(N.lib.lpg_fem_set_stream(e.handle, None))
    E = ctypes.c_double()

    def e2e_step():
        N.check(N.lib.lpg_fem_eval(e.handle, N.vptr(u_pin), N.MEM_HOST, ctypes.byref(E), N.vptr(g_pin), int(Exact),
                                   N.PRECISION_F64, N.LAYOUT_CSC, N.vptr(h_pin), N.MEM_HOST))

    for _ in range(2):
        e2e_step()
    k_e2e = max(3, min(args.steps, 10))
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        e2e_step()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world)
    e2e = {"value": whole_job_rate(T * k_e2e, e2e_s, world), "unit": "tets/s", "h2d_bytes_per_step": 8 * 3 * V,
           "d2h_bytes_per_step": 8 * 3 * V + 8 * e.nnz + 8, "steps": k_e2e,
           "timing": "wall clock around synchronous lpg_fem_eval calls (pinned host buffers, CSC layout)"}

    newton = None
    if not args.no_newton:
        try:
            newton = newton_times(e, g, torch)
        except Exception as exc:  # reported, not hidden
            newton = {"error": f"{type(exc).__name__}: {exc}"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(X, tets, theta, u_host)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "tets/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded structured five-tet box)",
            "config": workload_config(),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": gpu_launches,
            "clocks": clocks.summary(), "mixed_precision_kernel": mixed, "newton_time_to_1e-8": newton,
            "autotune": tuning_summary(e),
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run_kernels_only():
    """Three launches each of the FP64 exact, FP32 exact and FP64 projected assembly on the
    bench workload, nothing else (the command profiled by ncu)."""
    import torch

    from litepgo_b200 import energy, fem, workloads

    torch.cuda.set_device(0)
    g = workloads.gravity_box(N_CUBES, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    u = torch.as_tensor(state(g["X"]), device="cuda")
    for kind, prec in ((energy.HessianKind.Exact, "f64"), (energy.HessianKind.Exact, "mixed"),
                       (energy.HessianKind.Projected, "f64")):
        for _ in range(3):
            e.eval_device(u, gradient=True, hessian=kind, precision=prec)
    torch.cuda.synchronize()
    print("kernels ok")
    return 0


def run_newton_only(prec, iterations):
    """A Newton solve of the bench workload cut at `iterations` Newton iterations, run twice
    (the second with the PCG graph cached): a short command for ncu launch lists."""
    import scipy.sparse as sp
    import torch

    from litepgo_b200 import dof, energy, fem, solver, workloads

    torch.cuda.set_device(0)
    g = workloads.gravity_box(N_CUBES, seed=0)
    e = fem.VolumetricFemEnergyTetP1.from_arrays(g["X"], g["tets"], g["theta"])
    n = g["X"].size
    total = energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"]), 1.0)])
    fixed = dof.DofReduction(n, g["fixed"])
    x0 = torch.zeros(n, dtype=torch.float64, device="cuda")
    opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo", precision=prec,
                                max_iterations=iterations, cg_tolerance=1e-2, cg_max_iterations=20000)
    for _ in range(2):
        r = solver.newton_solve(total, fixed, x0, opts)
        print(json.dumps({"precision": prec, "status": r.status.name, "iterations": r.iterations,
                          "cg_iterations": int(r.cg_iterations), "seconds": r.seconds}), flush=True)
    return 0


def run_stress(steps):
    """The 128^3 compression stress case: per-result error of the mixed path against FP64,
    assembly GB/s of both kernels, and Newton time-to-1e-8 (relative gradient, Armijo) with the
    top and bottom faces held at the compressed state, mixed vs FP64. The Newton uses the
    projected Hessian until the gradient has fallen by 1e3, then the Exact one (exact_below): from
    this noisy state the projected Hessian alone converges only linearly near the solution, and
    the Exact one alone is indefinite far from it. Prints one JSON line."""
    import torch

    from litepgo_b200 import _native as N
    from litepgo_b200 import dof, energy, fem, solver, workloads

    torch.cuda.set_device(0)
    w = workloads.compressed_box(128, seed=0)
    X, tets, u_host = w["X"], w["tets"], w["u"]
    T, V = tets.shape[0], X.shape[0]
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, w["theta"])
    u = torch.as_tensor(u_host, device="cuda")
    Exact = energy.HessianKind.Exact
    E64, g64, H64 = e.eval_device(u, gradient=True, hessian=Exact, precision="f64")
    E32, g32, H32 = e.eval_device(u, gradient=True, hessian=Exact, precision="mixed")
    errors = {"energy": abs(E32 - E64) / abs(E64),
              "gradient": float((g32 - g64).abs().max() / g64.abs().max()),
              "hessian": float((H32.double() - H64).abs().max() / H64.abs().max())}
    del H32
    peak, _ = measured_peak()
    kernels = {}
    for prec, name, dt in ((N.PRECISION_F64, "f64", torch.float64), (N.PRECISION_MIXED, "mixed", torch.float32)):
        hess = H64 if prec == N.PRECISION_F64 else torch.empty(e.nnz, dtype=dt, device="cuda")
        ma, me = ctypes.c_double(), ctypes.c_double()
        N.check(N.lib.lpg_fem_set_stream(e.handle, ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        N.check(N.lib.lpg_fem_time_eval(e.handle, N.vptr(u), N.vptr(g64), int(Exact), prec, N.LAYOUT_BSR,
                                        N.vptr(hess), steps, 1, ctypes.byref(ma), ctypes.byref(me)))
        ab = algorithmic_bytes(T, V, e.nnzb, "f64" if name == "f64" else "f32")
        gbs = ab / (ma.value * 1e-3) / 1e9
        kernels[name] = {"kernel_ms": ma.value, "tets_per_s": T / (ma.value * 1e-3), "achieved_gbs": gbs,
                         "frac_of_measured_hbm": gbs / peak, "algorithmic_bytes": ab}
    del H64
    N.check(N.lib.lpg_fem_set_stream(e.handle, None))
    top_bottom = np.flatnonzero((X[:, 2] == 0.0) | (X[:, 2] == 1.0))
    fixed = dof.DofReduction(3 * V, (3 * top_bottom[:, None] + np.arange(3)).ravel())
    newton = {}
    for prec in ("mixed", "f64"):
        opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                    precision=prec, max_iterations=300, cg_tolerance=1e-2, cg_max_iterations=50000,
                                    exact_below=1e-3)
        r = solver.newton_solve(e, fixed, u, opts)
        newton[prec] = {"status": r.status.name, "seconds": r.seconds, "iterations": r.iterations,
                        "cg_iterations": int(r.cg_iterations), "energy": r.energy,
                        "relative_gradient": r.gradient_norm / max(r.gradient_norm0, 1e-300)}
        newton[prec + "_x"] = r.x
    xm, xf = newton.pop("mixed_x"), newton.pop("f64_x")
    newton["max_abs_diff_mixed_vs_f64"] = float((xm - xf).abs().max())
    if newton["mixed"]["seconds"] > 0:
        newton["speedup_mixed_vs_f64"] = newton["f64"]["seconds"] / newton["mixed"]["seconds"]
    print(json.dumps({"workload": "compressed box 128^3 cubes x 5 tets (V=2146689, T=10485760, nnzb=27608193), "
                                  "z scaled by 0.6 plus 0.05 h N(0,1) per vertex, det F in [0.2, 3.0], seed "
                                  f"{w['seed']}; Newton (projected, Exact below 1e-3 relative gradient): top and bottom faces "
                                  "held, interior relaxed",
                      "mixed_vs_f64_errors": errors, "assembly": kernels, "newton_time_to_1e-8": newton}), flush=True)
    return 0


def run_batch():
    """Config 3: 256 uneven boxes (cube counts per axis U{4..24}) solved as one batch by
    solver.batch_newton_solve (relative gradient 1e-8, Armijo; projected Hessian, Exact once every
    unfinished mesh's gradient has fallen by 1e3), mixed and FP64; meshes/s and the
    per-mesh p50 / p99 completion times, beside the same meshes solved one call each (a sample of
    32). Prints one JSON line."""
    import scipy.sparse as sp
    import torch

    from litepgo_b200 import dof, energy, fem, solver, workloads

    torch.cuda.set_device(0)
    b = workloads.batch_boxes(count=256, seed=0)
    X, tets, voff, eoff = b["X"], b["tets"], b["vertex_offsets"], b["element_offsets"]
    n = X.size

    def total_energy(Xs, ts, f):
        e = fem.VolumetricFemEnergyTetP1.from_arrays(Xs, ts, b["theta"])
        return energy.WeightedSumEnergy([(e, 1.0), (energy.QuadraticEnergy(sp.csc_matrix((f.size, f.size)), -f), 1.0)])

    union = total_energy(X, tets, b["f"])
    fixed = dof.DofReduction(n, b["fixed"])
    x0 = torch.as_tensor(b["u0"], device="cuda")
    out = {"workload": f"256 boxes, cube counts per axis U{{4..24}}, spacing 1/16, seed {b['seed']}: "
                       f"V={X.shape[0]}, T={tets.shape[0]} (mean {tets.shape[0] / 256:.0f} tets per mesh); "
                       "per-mesh affine state A = I + 0.1 N(0,1), bottom face fixed, gravity",
           "rule": "relative gradient 1e-8, Armijo, exact_below 1e-3, at most 400 Newton iterations"}
    for prec in ("mixed", "f64"):
        # Tall slender boxes collapse under their own weight far from their start (the oracle's
        # direct-solve Newton takes 84-99 iterations on them), hence the cap of 400.
        opts = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                    precision=prec, max_iterations=400, cg_tolerance=1e-2, exact_below=1e-3)
        warm = solver.NewtonOptions(gradient_tolerance=1e-8, stop_rule="relative", accept_rule="armijo",
                                    precision=prec, max_iterations=1, cg_tolerance=1e-2)
        solver.batch_newton_solve(union, voff, eoff, fixed, x0, warm)
        torch.cuda.synchronize()
        _, per, total = solver.batch_newton_solve(union, voff, eoff, fixed, x0, opts)
        t = np.array([p.seconds for p in per])
        it = np.array([p.iterations for p in per])
        tc = np.array([p.seconds for p in per if p.status == 0])
        out[prec] = {"seconds": total.seconds, "meshes_per_s": 256 / total.seconds,
                     "per_mesh_p50_s": float(np.percentile(t, 50)), "per_mesh_p99_s": float(np.percentile(t, 99)),
                     "converged_p50_s": float(np.percentile(tc, 50)), "converged_p99_s": float(np.percentile(tc, 99)),
                     "converged": int(sum(p.status == 0 for p in per)), "newton_iterations_max": int(it.max()),
                     "newton_iterations_p50": float(np.median(it)), "lockstep_cg_iterations": int(total.cg_iterations)}
        # The same meshes one call each (first 32): per-mesh seconds and the implied meshes/s.
        single = []
        for m in range(32):
            v0, v1, e0, e1 = voff[m], voff[m + 1], eoff[m], eoff[m + 1]
            fm = b["f"][3 * v0:3 * v1]
            fx = b["fixed"][(b["fixed"] >= 3 * v0) & (b["fixed"] < 3 * v1)] - 3 * v0
            em = total_energy(X[v0:v1], tets[e0:e1] - v0, fm)
            xm0 = x0[3 * v0:3 * v1].contiguous()
            solver.newton_solve(em, dof.DofReduction(3 * (v1 - v0), fx), xm0, warm)
            t0 = time.perf_counter()
            r = solver.newton_solve(em, dof.DofReduction(3 * (v1 - v0), fx), xm0, opts)
            single.append((time.perf_counter() - t0, int(r.status), r.iterations))
        out[prec]["one_call_per_mesh_sample"] = {
            "meshes": 32, "mean_s": float(np.mean([s_[0] for s_ in single])),
            "meshes_per_s": 1.0 / float(np.mean([s_[0] for s_ in single])),
            "converged": sum(s_[1] == 0 for s_ in single),
            "batch_statuses_of_these": [int(p.status) for p in per[:32]],
            "single_iterations": [s_[2] for s_ in single], "batch_iterations": [int(p.iterations) for p in per[:32]]}
    print(json.dumps(out), flush=True)
    return 0


def run_rows():
    """The widened rows on the bench mesh (64^3 gravity box): the plastic-field force VJP kernel
    (per element, device arrays) with its algorithmic bytes, the equilibrium adjoint in Fp, and
    VEG write / read of the mesh. Prints one JSON line."""
    import tempfile

    import scipy.sparse as sp
    import torch

    from litepgo_b200 import _native as N
    from litepgo_b200 import dof, energy, fem, mesh, solver, workloads

    torch.cuda.set_device(0)
    g = workloads.gravity_box(N_CUBES, seed=0)
    X, tets, theta = g["X"], g["tets"], g["theta"]
    T, V, n = tets.shape[0], X.shape[0], X.size
    rng = np.random.default_rng(21)
    Fp = np.stack([(np.eye(3) + 0.02 * rng.standard_normal((3, 3))).T.ravel() for _ in range(T)])
    e = fem.VolumetricFemEnergyTetP1.from_arrays(X, tets, theta, Fp=Fp)
    dev = torch.device("cuda", 0)
    u = torch.as_tensor(state(X), device=dev)
    w = torch.as_tensor(rng.standard_normal(n), device=dev)
    out = torch.empty(9 * T, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream()
    N.check(N.lib.lpg_fem_set_stream(e.handle, ctypes.c_void_p(stream.cuda_stream)))

    def vjp():
        N.check(N.lib.lpg_fem_force_vjp_fp(e.handle, N.vptr(u), N.vptr(w), N.MEM_DEVICE, 1, N.vptr(out)))

    for _ in range(3):
        vjp()
    k = 20
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(k):
        vjp()
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1) / k
    # Per element: tet indices 16, FP64 record 96, Fp^-1 72, 9 outputs 72; per vertex u and w.
    fp_bytes = T * (16 + 96 + 72 + 72) + V * 48
    peak, _ = measured_peak()
    fp_row = {"call_ms": ms, "tets_per_s": T / (ms * 1e-3), "algorithmic_bytes": fp_bytes,
              "achieved_gbs": fp_bytes / (ms * 1e-3) / 1e9, "frac_of_measured_hbm": fp_bytes / (ms * 1e-3) / 1e9 / peak,
              "timing": "CUDA events around 20 synchronous lpg_fem_force_vjp_fp calls (device arrays; each call "
                        "ends with its status read-back); working set ~350 MB > L2"}
    # Equilibrium adjoint in Fp at the gravity equilibrium of the plastic box.
    N.check(N.lib.lpg_fem_set_stream(e.handle, None))
    load = energy.QuadraticEnergy(sp.csc_matrix((n, n)), -g["f"])
    total = energy.WeightedSumEnergy([(e, 1.0), (load, 1.0)])
    fixed = dof.DofReduction(n, g["fixed"])
    opts = solver.NewtonOptions(gradient_tolerance=1e-10, stop_rule="relative", accept_rule="armijo",
                                max_iterations=100, cg_tolerance=1e-2, exact_below=1e-3)
    r = solver.newton_solve(total, fixed, np.zeros(n), opts)
    x = np.asarray(r.x)
    dLdx = rng.standard_normal(n)
    fixed_arr = np.ascontiguousarray(g["fixed"], dtype=np.int32)
    dFp = np.empty(9 * T)
    adj = {}
    for prec, name in ((N.PRECISION_F64, "f64"), (N.PRECISION_MIXED, "mixed")):
        t0 = time.perf_counter()
        N.check(N.lib.lpg_adjoint_fp(e.handle, N.vptr(x), N.vptr(dLdx), N.iptr(fixed_arr), int(fixed_arr.size),
                                     N.MEM_HOST, prec, 1e-10, 1, N.vptr(dFp), None))
        adj[name] = {"seconds": time.perf_counter() - t0, "norm": float(np.linalg.norm(dFp))}
    # VEG write / read of the mesh.
    with tempfile.TemporaryDirectory() as d:
        path = Path(d) / "box64.veg"
        t0 = time.perf_counter()
        mesh.write_veg(path, mesh.TetMesh(X, tets))
        tw = time.perf_counter() - t0
        size = path.stat().st_size
        t0 = time.perf_counter()
        back = mesh.read_veg(path)
        tr = time.perf_counter() - t0
        exact = bool(np.array_equal(back.positions, X) and np.array_equal(back.cells, tets))
    # Hex Q1 (GaussLegendre3D[2]) E + gradient + Exact Hessian on a 48^3 hex box.
    Xh, ch = mesh.make_hex_box(48)
    eh = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexQ1Basis, fem.GaussLegendre3D[2]].from_arrays(
        Xh, ch, np.array([1.4e5, 3.4e4]))
    uh = torch.as_tensor(state(Xh), device=dev)
    gh = torch.empty(Xh.size, dtype=torch.float64, device=dev)
    Hh = torch.empty(eh.nnz, dtype=torch.float64, device=dev)
    N.check(N.lib.lpg_fem_set_stream(eh.handle, ctypes.c_void_p(stream.cuda_stream)))
    ma, me = ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_time_eval(eh.handle, N.vptr(uh), N.vptr(gh), int(energy.HessianKind.Exact), N.PRECISION_F64,
                                    N.LAYOUT_BSR, N.vptr(Hh), 10, 1, ctypes.byref(ma), ctypes.byref(me)))
    pa, pe, ra, re = ctypes.c_double(), ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_time_eval(eh.handle, N.vptr(uh), N.vptr(gh), int(energy.HessianKind.Projected),
                                    N.PRECISION_F64, N.LAYOUT_BSR, N.vptr(Hh), 10, 1, ctypes.byref(pa), ctypes.byref(pe)))
    rest = torch.zeros_like(uh)  # every quadrature tangent semi-definite: no element needs the eigen-projection
    N.check(N.lib.lpg_fem_time_eval(eh.handle, N.vptr(rest), N.vptr(gh), int(energy.HessianKind.Projected),
                                    N.PRECISION_F64, N.LAYOUT_BSR, N.vptr(Hh), 10, 1, ctypes.byref(ra), ctypes.byref(re)))
    hex_row = {"mesh": f"hex box 48^3 ({ch.shape[0]} hexes, {Xh.shape[0]} vertices, nnzb {eh.nnzb}), 8 points",
               "element_pass_and_gather_ms": ma.value, "eval_ms": me.value, "hexes_per_s": ch.shape[0] / (me.value * 1e-3),
               "projected": {"element_pass_projection_and_gather_ms": pa.value, "eval_ms": pe.value,
                             "hexes_per_s": ch.shape[0] / (pe.value * 1e-3),
                             "at_rest_eval_ms": re.value, "at_rest_hexes_per_s": ch.shape[0] / (re.value * 1e-3)},
               "timing": "lpg_fem_time_eval: CUDA events, L2 flushed between launches, FP64 E + gradient + BSR "
                         "(Exact, and Projected: per-element 24x24 eigen-projection)"}
    # Tricubic Hermite hexes (GaussLegendre3D[2]) E + gradient + Exact Hessian on a 12^3 box.
    Xm, cm = mesh.make_hex_box(12)
    em = fem.VolumetricFemEnergy[fem.NeoHookean, fem.HexHermiteBasis, fem.GaussLegendre3D[2]].from_arrays(
        Xm, cm, np.array([1.4e5, 3.4e4]))
    um = torch.as_tensor(0.005 * np.random.default_rng(3).standard_normal(em.num_dofs), device=dev)
    gm = torch.empty(em.num_dofs, dtype=torch.float64, device=dev)
    Hm = torch.empty(em.nnz, dtype=torch.float64, device=dev)
    N.check(N.lib.lpg_fem_set_stream(em.handle, ctypes.c_void_p(stream.cuda_stream)))
    ha, he = ctypes.c_double(), ctypes.c_double()
    N.check(N.lib.lpg_fem_time_eval(em.handle, N.vptr(um), N.vptr(gm), int(energy.HessianKind.Exact), N.PRECISION_F64,
                                    N.LAYOUT_BSR, N.vptr(Hm), 10, 1, ctypes.byref(ha), ctypes.byref(he)))
    hermite_row = {"mesh": f"Hermite hex box 12^3 ({cm.shape[0]} hexes, {em.num_dofs} DOFs, nnzb {em.nnzb}), 8 points",
                   "element_pass_and_gather_ms": ha.value, "eval_ms": he.value,
                   "hexes_per_s": cm.shape[0] / (he.value * 1e-3),
                   "timing": "lpg_fem_time_eval: CUDA events, L2 flushed between launches, FP64 E + gradient + Exact BSR"}
    line = {"rows": "plastic-field force VJP, adjoint in Fp, VEG I/O, hex Q1, Hermite hex", "config": workload_config(),
            "hex_q1": hex_row, "hex_hermite": hermite_row,
            "fp_vjp": fp_row, "newton_with_fp": {"status": r.status.name, "iterations": r.iterations, "seconds": r.seconds},
            "adjoint_fp": adj,
            "veg": {"bytes": size, "write_s": tw, "read_s": tr, "read_mb_per_s": size / tr / 1e6,
                    "write_mb_per_s": size / tw / 1e6, "round_trip_exact": exact}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-newton", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--only-kernels", action="store_true",
                    help="run 3 evaluations of each assembly variant and exit (a short command for ncu)")
    ap.add_argument("--only-newton", choices=("mixed", "f64"), default=None,
                    help="run a Newton solve cut at --newton-iterations iterations and exit (for ncu launch lists)")
    ap.add_argument("--newton-iterations", type=int, default=2)
    ap.add_argument("--stress", action="store_true",
                    help="run the 128^3 compression stress case (errors, assembly GB/s, Newton) and exit")
    ap.add_argument("--rows", action="store_true",
                    help="time the plastic-field VJP, the adjoint in Fp and VEG I/O on the bench mesh and exit")
    ap.add_argument("--batch", action="store_true",
                    help="run the 256-mesh batched Newton (meshes/s, per-mesh p50/p99) and exit")
    args = ap.parse_args()
    if args.rows:
        return run_rows()
    if args.batch:
        return run_batch()
    if args.stress:
        return run_stress(max(args.steps, 3))
    if args.only_kernels:
        return run_kernels_only()
    if args.only_newton:
        return run_newton_only(args.only_newton, args.newton_iterations)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
