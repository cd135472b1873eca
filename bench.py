#!/usr/bin/env python3
"""Benchmark: SBDF3 steps/s of the rotational plane-Couette KMM step.

Workload (one "step" = one steady SBDF3 step of the whole field): the Couette
DNS configuration, 65 x 64 x 64 (Chebyshev wall-normal x Fourier x Fourier,
3/2 dealiasing), Re = 1000, dt = 0.01, seeded divergence-free perturbation of
energy 1e-4 (jaxfun_b200.workloads).  Single-GPU problem: with --gpus N every
rank advances its own replica (weak scaling, no collective on the data path).

Default arm (--impl b200), run for both forms of the step (--precision both):
the mixed form (complex64 periodic transforms and rotational products, FP64
Shen operators, right-hand sides and solves) is the headline value, the FP64
form is reported beside it, and the per-field relative L2 distance between
the two after 100 and 1000 steps of the same workload is stated in the line.
Each form times K steady steps, each one CUDA-graph launch
bracketed by CUDA events on the launching stream (a 256 MiB memset before
each step flushes the 126 MB L2 outside the events); a second, untimed pass
through ``jfb_kmm_timed_steps`` gives per-kernel times (events around every
launch); reports the per-kernel roofline of the dominant kernel, the
back-to-back CUDA-graph throughput, an end-to-end figure through the public
``solve`` API with pinned host buffers, and the CPU oracle on the host cores.
Further blocks (each with a --no-... switch): the adjoint and minimal-seed
ascent, the MHD ensemble, the 2-D Helmholtz solve, the linear-stability tools
(growth-rate map and optimal-growth scan), the larger grids and the
reference's default (gradient) form with its integrators.

Reference arm (--impl reference): the reference (JAX) cannot be installed
here, so the reference's CPU algorithm is timed through the NumPy/SciPy
restatement in oracle/ on all host cores, on the same workload.
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SBDF3 steps/s at 65×64×64 on 1 B200: mixed vs FP64 form at stated err, vs CPU"
UNIT = "steps/s"
RE, DT, ENERGY = 1000.0, 0.01, 1.0e-4
HBM_FALLBACK_GBS = 6650.0
FLUSH_BYTES = 256 << 20
BLOCK = 25  # reference rollout block (production/benchmark.py: rollout_steps)


def parse_args(argv=None):
    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=20)
    p.add_argument("--impl", choices=("b200", "reference"), default="b200")
    p.add_argument("--precision", choices=("both", "fp64", "mixed"), default="both",
                   help="both: headline = mixed form, FP64 form and the mixed-vs-FP64 "
                        "error in the same line")
    p.add_argument("--grid", default="65,64,64")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-adjoint", action="store_true",
                   help="skip the adjoint / minimal-seed block")
    p.add_argument("--adjoint-steps", type=int, default=200)
    p.add_argument("--ascent-iterations", type=int, default=20)
    p.add_argument("--no-ensemble", action="store_true",
                   help="skip the MHD ensemble block")
    p.add_argument("--ensemble-members", type=int, default=32)
    p.add_argument("--no-helmholtz", action="store_true",
                   help="skip the 2-D Helmholtz block")
    p.add_argument("--no-linear", action="store_true",
                   help="skip the linear-stability / transient-growth block")
    p.add_argument("--no-default-form", action="store_true",
                   help="skip the gradient-form (the reference's default) timing block")
    p.add_argument("--no-sizes", action="store_true",
                   help="skip the 97^3 / 129^3 mixed-vs-FP64 block")
    p.add_argument("--no-autotune", action="store_true",
                   help="time the default kernel variant instead of the autotuner's choice")
    return p.parse_args(argv)


def grid_of(args):
    return tuple(int(v) for v in args.grid.split(","))


def domain():
    return ((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi))


def workload_desc(grid):
    """The benchmark configuration (identical in both arms)."""
    nx, ny, nz = grid
    return {
        "workload": (
            f"plane Couette KMM SBDF3 rotational step {nx}x{ny}x{nz} "
            f"(Chebyshev x Fourier x Fourier, 3/2 dealiasing), Re={RE:g}, dt={DT:g}, "
            f"seeded divergence-free perturbation, energy {ENERGY:g}"
        ),
        "grid": list(grid),
        "forms": "mixed (complex64 transforms and products, FP64 operators and solves) "
                 "as the headline; FP64 alongside",
        "parallelism": "replicas",
    }


def stage_bytes(grid, my, precision="fp64"):
    """Algorithmic HBM bytes per launch of each kernel and per step, in the
    stage model: Hermitian half spectra H = Nz/2 + 1, E_s = Nx Ny H,
    E_m = Nx My H, factors regenerated (0 B), each array read once and written
    once.  FP64: 16 B per complex value everywhere.  Mixed form: 16 B for the
    coefficient-space state, history and right-hand sides, 8 B for the
    x-physical fields and the periodic-axis stages."""
    nx, ny, nz = grid
    H = nz // 2 + 1
    Es, Em = nx * ny * H, nx * my * H
    hi, lo = 16, (8 if precision == "mixed" else 16)
    return {
        # reads: H 3 E_s (lo) + solution levels 6 E_s + nonlinear levels 4 E_s;
        # writes: new (u0, g) 2 E_s + N 2 E_s + six x-physical fields 6 E_s (lo)
        "pencil_stage": 14 * Es * hi + 9 * Es * lo,
        "y_backward": (6 * Es + 6 * Em) * lo,
        "z_cross": 9 * Em * lo,
        "y_forward": (3 * Em + 3 * Es) * lo,
        # fused plane transforms: reads X (6 E_s), writes HX (3 E_s)
        "plane_transforms": 9 * Es * lo,
        # canonical whole-step figure: FP64 (43 E_s + 18 E_m) x 16 B; mixed
        # 544 E_s + 144 E_m bytes
        "step": (43 * Es + 18 * Em) * 16 if precision != "mixed" else 544 * Es + 144 * Em,
    }


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback"


def dram_traffic(kernel, precision, grid):
    """Per-launch DRAM bytes of `kernel` on `grid` from the committed ncu
    summaries (null when that kernel and grid were not captured)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
    except (OSError, ValueError):
        return None
    return t.get("x".join(str(n) for n in grid), {}).get(f"{kernel}/{precision}")


class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.file = None

    def start(self):
        try:
            self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.index)],
                stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, ValueError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        rows = [r.strip().split(",") for r in self.file if r.strip()]
        os.unlink(self.file.name)
        sm, smax, reasons = [], None, set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                smax = float(r[2])
                for name, v in zip(names, r[5:9], strict=False):
                    if v.strip().lower() in ("active", "1"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_oracle_rate(fields, grid, seconds, threads):
    """Steady SBDF3 steps/s of the oracle (NumPy/SciPy restatement of the
    reference algorithm) on the host cores; a bounded sample."""
    from oracle import kmm as ok

    ok.set_workers(threads)
    o = ok.PlaneCouetteOracle(N=grid, Re=RE, dt=DT, domain=domain(),
                              perturbation_amplitude=0.0)
    st = o.state_from_physical(tuple(f.astype(complex) for f in fields))
    st = o.step(o.step(st))  # IMEXRK3 startup, not timed
    st = o.step(st)          # warm
    n, t0 = 0, time.perf_counter()
    while True:
        st = o.step(st)
        n += 1
        if n >= 3 and time.perf_counter() - t0 >= seconds:
            break
    dt = time.perf_counter() - t0
    return n / dt, n


def _single_threaded_worker():
    """Pool initializer: one BLAS / FFT thread per worker process (set before
    the worker imports numpy)."""
    for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS"):
        os.environ[k] = "1"


def _helmholtz_cpu_worker(seconds):
    """Oracle 2-D Helmholtz solves of the seeded 64 x 64 forcing for about
    `seconds` in one process: (solves, elapsed seconds)."""
    from jaxfun_b200.workloads import helmholtz2d_forcing
    from oracle import kmm as ok

    fh = helmholtz2d_forcing((64, 64), seed=1)
    ok.helmholtz2d_solve(fh)  # warm
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        ok.helmholtz2d_solve(fh)
        n += 1
    return n, time.perf_counter() - t0


def helmholtz_cpu_rate(threads, seconds=2.0):
    """Throughput of the oracle's 2-D Helmholtz solve on all host cores: one
    spawned process per core, each solving the same seeded problem for about
    `seconds`; returns (microseconds per solve at that throughput, solves)."""
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor

    with ProcessPoolExecutor(max_workers=threads, mp_context=mp.get_context("spawn"),
                             initializer=_single_threaded_worker) as pool:
        res = list(pool.map(_helmholtz_cpu_worker, [seconds] * threads))
    rate = sum(n / t for n, t in res)
    return 1e6 / rate, sum(n for n, _ in res)


def max_over_ranks(value: float, device) -> float:
    """Max of a per-rank scalar over the process group (identity if none)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def reference_arm(args):
    grid = grid_of(args)
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from jaxfun_b200.workloads import couette_perturbation_fields

    fields = couette_perturbation_fields(grid, domain())
    threads = host_threads()
    # energy normalisation is linear: scale with the oracle's own projection
    from oracle import kmm as ok

    ok.set_workers(threads)
    o = ok.PlaneCouetteOracle(N=grid, Re=RE, dt=DT, domain=domain())
    e = o.diagnostics(o.state_from_physical(tuple(f.astype(complex) for f in fields)))["Epert"]
    s = math.sqrt(ENERGY / e)
    fields = tuple(f * s for f in fields)
    per_step = max(3.0, args.cpu_seconds / max(1, args.steps))
    rates = []
    for _ in range(max(1, min(args.warmup, 1))):
        cpu_oracle_rate(fields, grid, 1.0, threads)
    for _ in range(max(1, min(args.steps, 3))):
        r, _ = cpu_oracle_rate(fields, grid, per_step, threads)
        rates.append(r)
    value = statistics.median(rates)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1000.0 / value,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": workload_desc(grid),
        "l2": "n/a (host CPU, FP64 restatement)",
        "cpu_baseline": {
            "value": value, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{len(rates)} samples of >= {per_step:.1f} s of steady SBDF3 steps "
                      "of the oracle restatement (reference JAX not installable: no jax/jaxlib "
                      "in the image, no network)",
        },
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def main(argv=None):
    args = parse_args(argv)
    if args.impl == "reference":
        return reference_arm(args)

    import ctypes

    import torch
    import torch.distributed as dist

    from jaxfun_b200 import _lib
    from jaxfun_b200.kmm import KMMState, PlaneCouetteFluctuation
    from jaxfun_b200.workloads import couette_perturbation_fields, scale_to_energy

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120),
                                device_id=dev)
    grid = grid_of(args)

    stream = torch.cuda.current_stream(dev)
    fields0 = couette_perturbation_fields(grid, domain())
    flush = torch.empty(FLUSH_BYTES, dtype=torch.uint8, device=dev)

    def measure(precision):
        """Timed steady steps, per-kernel breakdown, graph replay and the
        end-to-end figure of one form on the seeded workload."""
        solver = PlaneCouetteFluctuation(N=grid, domain=domain(), Re=RE, dt=DT,
                                         precision=precision, device=dev,
                                         time_integrator="SBDF3", nonlinear_form="rotational")
        info = solver.info()
        e0 = solver.diagnostics(solver.state_from_physical(fields0))["Epert"]
        fields = scale_to_energy(fields0, e0, ENERGY)
        state = solver.state_from_physical(fields)
        # kernel variant: the autotuner's choice for this grid and form
        # (CUDA-event timing of graph-replayed steps, untimed here)
        tuned = solver.autotune(state, steps=20, cache=False) if not args.no_autotune else None
        # warm-up: startup + W steady steps (graph replay), device resident
        state = solver.solve(state, 2 + max(3, args.warmup))
        torch.cuda.synchronize(dev)
        # timed region: K steady steps, each one CUDA-graph launch (the
        # production path) bracketed by events; a 256 MiB memset before each
        # step flushes the 126 MB L2 outside the events
        starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
        sampler = ClockSampler(local)
        sampler.start()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        for i in range(args.steps):
            flush.fill_(i & 0xFF)
            starts[i].record(stream)
            solver.advance_resident(1)
            ends[i].record(stream)
        torch.cuda.synchronize(dev)
        if world > 1:
            dist.barrier()
        clocks = sampler.stop()
        solver._current = None
        step_ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends, strict=True))
        t_step = max_over_ranks(step_ms / max(1, args.steps), dev)

        # per-kernel breakdown (diagnostic, outside the timed region): events
        # around each kernel launch, L2 flushed before each step; every
        # interval also holds one kernel launch latency
        kms = (ctypes.c_double * 4)()
        sms = ctypes.c_double()
        kb_steps = min(args.steps, 50)
        _lib.call("jfb_kmm_timed_steps", solver._plan, kb_steps, flush.data_ptr(), FLUSH_BYTES,
                  kms, ctypes.byref(sms), ctypes.c_void_p(stream.cuda_stream))
        torch.cuda.synchronize(dev)
        solver._current = None
        info = solver.info()  # launches per step of the selected variant
        if info.launches_per_step == 2:  # pencil stage + fused plane transforms
            names = ("pencil_stage", "plane_transforms")
        else:
            names = ("pencil_stage", "y_backward", "z_cross", "y_forward")
        kernel_avg = {k: kms[i] / kb_steps for i, k in enumerate(names)}

        # back-to-back graph replay (L2 stays warm between steps)
        g_steps = max(10, args.steps)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        solver.advance_resident(g_steps)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        graph_ms = max_over_ranks(e0.elapsed_time(e1) / g_steps, dev)

        # end to end through the public API with pinned host buffers
        cur = solver._fetch(2.0)

        def host_copy(t):
            h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
            h.copy_(t)
            return h

        def tree(st, fn):
            lv = lambda x: tuple(fn(t) for t in x)  # noqa: E731
            return KMMState(u=lv(st.u), g=fn(st.g), nonlinear_old=lv(st.nonlinear_old),
                            nonlinear_older=lv(st.nonlinear_older),
                            solution_old=lv(st.solution_old),
                            solution_older=lv(st.solution_older),
                            history_steps=st.history_steps)

        host_state = tree(cur, host_copy)
        state_bytes = sum(t.numel() * t.element_size() for t in
                          (*host_state.u, host_state.g, *host_state.nonlinear_old,
                           *host_state.nonlinear_older, *host_state.solution_old,
                           *host_state.solution_older))
        host_out = tree(cur, lambda t: torch.empty(t.shape, dtype=t.dtype, pin_memory=True))
        diag_host = torch.empty(8, dtype=torch.float64, pin_memory=True)
        blocks = max(1, min(4, args.steps // BLOCK))

        def e2e_block(hs):
            dstate = tree(hs, lambda t: t.to(dev, non_blocking=True))
            out = solver.solve(dstate, BLOCK)
            diag = solver.diagnostics_tensor(out)
            for src, dst in zip((*out.u, out.g, *out.nonlinear_old, *out.nonlinear_older,
                                 *out.solution_old, *out.solution_older),
                                (*host_out.u, host_out.g, *host_out.nonlinear_old,
                                 *host_out.nonlinear_older, *host_out.solution_old,
                                 *host_out.solution_older), strict=True):
                dst.copy_(src, non_blocking=True)
            diag_host.copy_(diag, non_blocking=True)
            return host_out

        # one untimed block first (allocator and first-use costs), from the
        # same host state as the timed blocks
        e2e_block(host_state)
        torch.cuda.synchronize(dev)
        solver._current = None
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x0.record(stream)
        hs = host_state
        for _ in range(blocks):
            hs = e2e_block(hs)
        x1.record(stream)
        torch.cuda.synchronize(dev)
        e2e_ms = max_over_ranks(x0.elapsed_time(x1) / (blocks * BLOCK), dev)
        final_diag = dict(zip(solver.DIAGNOSTIC_NAMES, diag_host.tolist(), strict=True))

        sb = stage_bytes(grid, info.my, precision)
        peak, peak_kind = measured_peak()
        dom = max(kernel_avg, key=kernel_avg.get)
        dom_ms = kernel_avg[dom]
        achieved = sb[dom] / (dom_ms * 1e-3) / 1e9
        step_ach = sb["step"] / (t_step * 1e-3) / 1e9
        return {
            "value": world * 1000.0 / t_step, "ms_per_step": t_step,
            "roofline": {
                "bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_kind": f"of {peak_kind}",
                "traffic": dram_traffic(dom, precision, grid),
                "algorithmic_bytes_per_launch": sb[dom], "launch_ms": dom_ms,
            },
            "step_roofline": {
                "algorithmic_bytes": sb["step"], "achieved": step_ach, "peak": peak,
                "unit": "GB/s", "frac": step_ach / peak, "peak_kind": f"of {peak_kind}",
            },
            "kernel_ms": kernel_avg,
            "graph_l2_resident": {"ms_per_step": graph_ms, "value": world * 1000.0 / graph_ms},
            "e2e": {
                "value": world * 1000.0 / e2e_ms, "unit": UNIT,
                "h2d_bytes_per_step": state_bytes / BLOCK,
                "d2h_bytes_per_step": (state_bytes + 64) / BLOCK,
                "path": f"solve(state, {BLOCK}) per block with pinned-host state in/out and "
                        "diagnostics read back",
            },
            "gpu_launches": solver.info().launches_per_step * args.steps,
            "autotune": tuned,
            "clocks": clocks,
            "final_diagnostics": final_diag,
            "device_bytes": info.device_bytes,
            "fields": fields,
        }

    def mixed_error():
        """Per-field relative L2 of the mixed form against the FP64 form after
        100 and 1000 steps from the same FP64-projected initial state."""
        g64 = PlaneCouetteFluctuation(N=grid, domain=domain(), Re=RE, dt=DT, device=dev,
                                      time_integrator="SBDF3", nonlinear_form="rotational")
        g32 = PlaneCouetteFluctuation(N=grid, domain=domain(), Re=RE, dt=DT,
                                      precision="mixed", device=dev,
                                      time_integrator="SBDF3", nonlinear_form="rotational")
        e0 = g64.diagnostics(g64.state_from_physical(fields0))["Epert"]
        f = scale_to_energy(fields0, e0, ENERGY)
        a, b = g64.state_from_physical(f), g32.state_from_physical(f)
        out, done = {}, 0
        for n in (100, 1000):
            a, b = g64.solve(a, n - done), g32.solve(b, n - done)
            done = n
            errs = {}
            for name, x, y in zip(("u0", "u1", "u2", "g"), (*b.u, b.g), (*a.u, a.g), strict=True):
                errs[name] = float(torch.linalg.norm(x - y) / torch.linalg.norm(y))
            num = sum(float(torch.linalg.norm(x - y)) ** 2 for x, y in zip((*b.u, b.g), (*a.u, a.g)))
            den = sum(float(torch.linalg.norm(y)) ** 2 for y in (*a.u, a.g))
            errs["state"] = math.sqrt(num / den)
            out[f"after_{n}_steps"] = errs
        return out

    def adjoint_block():
        """The adjoint / minimal-seed workload: gain E(T)/E(0) over
        --adjoint-steps FP64 SBDF3 steps of the same Couette problem, its
        gradient by the hand-written adjoint (recompute checkpoint every 20
        steps), central FD (eps 1e-6) along 8 seeded divergence-free
        directions (seeds 200..207), then --ascent-iterations projected-gradient
        ascent iterations at fixed initial energy 1e-4."""
        from jaxfun_b200 import minimal_seed as ms

        T, ck = args.adjoint_steps, 20
        g64 = PlaneCouetteFluctuation(N=grid, domain=domain(), Re=RE, dt=DT, device=dev,
                                      time_integrator="SBDF3", nonlinear_form="rotational")
        e0 = g64.diagnostics(g64.state_from_physical(fields0))["Epert"]
        x0 = ms._primary(g64.state_from_physical(scale_to_energy(fields0, e0, ENERGY)))
        ms.gain_and_gradient(g64, x0, 4, checkpoint=2)  # operators and bands, untimed
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        gain_f, _ = ms.gain_and_gradient(g64, x0, T, checkpoint=ck, with_gradient=False)
        torch.cuda.synchronize(dev)
        t1 = time.perf_counter()
        gain, grad = ms.gain_and_gradient(g64, x0, T, checkpoint=ck)
        torch.cuda.synchronize(dev)
        t2 = time.perf_counter()
        fd = []
        for m in range(8):
            f = couette_perturbation_fields(grid, domain(), seeds=(200 + m, 300 + m))
            d = ms._primary(g64.state_from_physical(f))
            d = ms.tree_scale(d, ms.tree_l2_norm(x0) / ms.tree_l2_norm(d))
            eps = 1e-6
            jp = ms.perturbation_gain(g64, ms.tree_add_scaled(x0, d, eps), T)
            jm = ms.perturbation_gain(g64, ms.tree_add_scaled(x0, d, -eps), T)
            fdv = (jp - jm) / (2 * eps)
            adj = ms.jax_complex_directional_derivative(grad, d)
            fd.append({"seed": 200 + m, "adjoint": adj, "fd": fdv,
                       "rel_err": abs(adj - fdv) / max(abs(fdv), 1e-300)})
        t3 = time.perf_counter()
        _, hist = ms.minimal_seed_ascent(g64, x0, target_energy=ENERGY, steps=T,
                                         iterations=args.ascent_iterations, step_size=1.0,
                                         checkpoint=ck)
        torch.cuda.synchronize(dev)
        t4 = time.perf_counter()
        return {
            "workload": f"{T} FP64 SBDF3 steps (2 IMEXRK3 startup) of the Couette workload, "
                        f"gain E(T)/E(0), checkpoint every {ck} steps",
            "gain": gain,
            "forward_s": t1 - t0,
            "gain_and_gradient_s": t2 - t1,
            "gradient_over_forward": (t2 - t1) / max(t1 - t0, 1e-12),
            "fd_check": {"eps": 1e-6, "directions": fd,
                         "max_rel_err": max(r["rel_err"] for r in fd)},
            "fd_s": t3 - t2,
            "ascent": {
                "iterations": len(hist),
                "accepted": sum(1 for h in hist if h.accepted),
                "gain_first": hist[0].gain if hist else None,
                "gain_last": hist[-1].gain if hist else None,
                "gains": [h.gain for h in hist],
                "seconds": t4 - t3,
            },
            "reference_jax_grad": "unavailable: jax is not installed on this host",
        }

    def ensemble_block():
        """The batched MHD ensemble workload: --ensemble-members members with
        wall-normal sizes cycling 33, 49, 65 x 64 x 64 Fourier modes, Re = Rm
        = 1000, imposed field B0 = 0.1 e_z, base flow U_b = x, seeded
        divergence-free perturbations of u and b (energies 1e-4 each); one
        CUDA graph per ensemble step.  The headline form is the mixed one
        (complex64 periodic transforms, FP64 solves); the FP64 form is timed
        beside it, and the two forms' per-field distance after the timed
        steps is reported."""
        from jaxfun_b200.mhd import Ensemble, MHDState, PlaneCouetteMRIShearpy

        sizes = (33, 49, 65)
        K = max(10, min(args.steps, 100))
        warm = 2 + max(3, args.warmup)
        states = []

        def build(precision):
            members = []
            for m in range(args.ensemble_members):
                N = (sizes[m % 3], grid[1], grid[2])
                sv = PlaneCouetteMRIShearpy(N=N, domain=domain(), Re=RE, Rm=RE, omega=0.0,
                                            shear_rate=-1.0, background_b=(0.0, 0.0, 0.1),
                                            dt=DT, precision=precision, device=dev)
                if len(states) <= m:
                    fu = couette_perturbation_fields(N, domain(), seeds=(100 + m, 1100 + m))
                    e_u = sv.diagnostics(sv.state_from_physical(fu))["Epert"]
                    flow = sv.state_from_physical(scale_to_energy(fu, e_u, ENERGY))
                    fa = couette_perturbation_fields(N, domain(), seeds=(2100 + m, 3100 + m))
                    A = sv._A_state_from_physical(fa)
                    e_b = sv.diagnostics(MHDState(flow=flow, A=A))["Emag"]
                    A = tuple(a * math.sqrt(ENERGY / e_b) for a in A)
                    states.append(MHDState(flow=flow, A=A))
                members.append(sv)
            return members

        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def timed(members, mode=None):
            """ms per ensemble step of the members (JFB200_ENSEMBLE=mode if
            given), after the same warm-up from the same states."""
            if mode is not None:
                os.environ["JFB200_ENSEMBLE"] = mode
            try:
                ens = Ensemble(members)
            finally:
                os.environ.pop("JFB200_ENSEMBLE", None)
            ens.load(states)
            ens.advance_resident(warm)
            torch.cuda.synchronize(dev)
            e0.record(stream)
            ens.advance_resident(K)
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return ens, e0.elapsed_time(e1) / K

        mixed = build("mixed")
        fp64 = build("fp64")
        ens, ms_step = timed(mixed)
        launches = ens.launches_per_step
        # the two forms after the same warm + K steps from the same states
        s32 = [m._fetch_mhd(2.0) for m in mixed[:3]]
        ens64, ms64 = timed(fp64)
        s64 = [m._fetch_mhd(2.0) for m in fp64[:3]]
        dist = {}
        for a, b, n in zip(s32, s64, sizes, strict=True):
            fa = (*a.flow.u, a.flow.g, *a.A)
            fb = (*b.flow.u, b.flow.g, *b.A)
            names = ("u0", "u1", "u2", "g", "Ax", "Ay", "Az")
            dist[f"N={n}"] = {k: float((x - y).norm() / y.norm())
                              for k, x, y in zip(names, fa, fb, strict=True)}
        diags = [m.diagnostics(s) for m, s in zip(mixed[:3], s32, strict=True)]
        # the other forms: every member on its own stream (the form of plans
        # that cannot batch) and all members in one group
        others = {}
        if ens.batched:
            others = {"one_stream_per_member": {"ms_per_ensemble_step": timed(mixed, "streams")[1]},
                      "one_group": {"ms_per_ensemble_step": timed(mixed, "batched")[1]},
                      "fp64_one_stream_per_member": {
                          "ms_per_ensemble_step": timed(fp64, "streams")[1]}}
        # stage model of one MHD member step: 91 E_s + 36 E_m complex values;
        # FP64 16 B each, mixed: the 36 E_s and 36 E_m values of the transform
        # arrays (X, Y, HZ, HX) at 8 B, the rest at 16 B
        bytes64 = bytes32 = 0
        for m in mixed:
            nx, ny, nz = m.N
            H = nz // 2 + 1
            Es, Em = nx * ny * H, nx * m.info().my * H
            bytes64 += (91 * Es + 36 * Em) * 16
            bytes32 += 1168 * Es + 288 * Em
        peak, peak_kind = measured_peak()

        def roof(b, ms):
            a = b / (ms * 1e-3) / 1e9
            return {"bound": "hbm", "achieved": a, "peak": peak, "unit": "GB/s",
                    "frac": a / peak, "peak_kind": f"of {peak_kind}",
                    "algorithmic_bytes_per_ensemble_step": b}

        return {
            "workload": f"{len(mixed)} MHD members, N cycling {sizes} x {grid[1]} x {grid[2]}, "
                        "Re = Rm = 1000, B0 = 0.1 e_z, u and b perturbation energies 1e-4",
            "members": len(mixed),
            "form": "mixed: complex64 periodic transforms and products, FP64 operators, "
                    "solves and state",
            "ms_per_ensemble_step": ms_step,
            "member_steps_per_s": len(mixed) * 1000.0 / ms_step,
            "steps": K,
            "gpu_launches_per_step": launches,
            "roofline": roof(bytes32, ms_step),
            "fp64": {"ms_per_ensemble_step": ms64,
                     "member_steps_per_s": len(fp64) * 1000.0 / ms64,
                     "roofline": roof(bytes64, ms64)},
            "mixed_vs_fp64_rel_l2": {"after_steps": warm + K, "members": dist},
            "other_forms": others,
            "launch": ("one CUDA graph per ensemble step: five launches per wall-normal size, "
                       "one per stage over that size's members' tiles, the sizes on parallel "
                       "branches" if ens.batched else
                       "one CUDA graph per ensemble step, one stream per member"),
            "l2": "not flushed: the ensemble's state exceeds L2",
            "device_bytes": sum(m.info().device_bytes for m in mixed),
            "sample_diagnostics": [{k: d[k] for k in ("Epert", "Emag", "divB_L2")} for d in diags],
        }

    def helmholtz_block():
        """The 2-D Helmholtz case: -lap u + u = f on 64 Chebyshev-Dirichlet x
        64 Fourier modes, seeded forcing; one solve = backward of f, scalar
        products, per-mode banded solves, backward of u.  Accuracy from a
        manufactured solution (f built from random coefficients of u with
        numpy's Chebyshev derivative), time per solve with CUDA events."""
        import numpy as np
        from numpy.polynomial import chebyshev as npc

        from jaxfun_b200.tps import Helmholtz2D
        from jaxfun_b200.workloads import helmholtz2d_forcing

        N = (64, 64)
        h = Helmholtz2D(N, device=dev)
        f_hat = torch.from_numpy(helmholtz2d_forcing(N, seed=1)).to(dev)
        rng = np.random.default_rng(2)
        uh = rng.standard_normal((N[0] - 2, N[1])) + 1j * rng.standard_normal((N[0] - 2, N[1]))
        uh[:, N[1] // 2] = 0
        uo = np.zeros((N[0], N[1]), dtype=complex)
        uo[:-2] += uh
        uo[2:] -= uh
        d2 = np.zeros_like(uo)
        d2[: N[0] - 2] = npc.chebder(uo, 2, axis=0)
        k = np.fft.fftfreq(N[1], 1.0 / N[1])
        fm = -d2 + (k[None, :] ** 2 + 1.0) * uo
        got = h.solve_coefficients(h.TC.backward(torch.from_numpy(fm).to(dev))).cpu().numpy()
        err = float(np.linalg.norm(got - uh) / np.linalg.norm(uh))
        for _ in range(5):
            h(f_hat)
        torch.cuda.synchronize(dev)
        K = 200
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(K):
            u = h(f_hat)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        us = e0.elapsed_time(e1) * 1000.0 / K
        for _ in range(5):
            h.separate(f_hat)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(K):
            h.separate(f_hat)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        us_sep = e0.elapsed_time(e1) * 1000.0 / K
        graph, f_in, _ = h.graphed(f_hat)
        for _ in range(3):
            graph.replay()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(K):
            graph.replay()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        us_graph = e0.elapsed_time(e1) * 1000.0 / K
        out = {
            "workload": "-lap u + u = f, 64 Chebyshev-Dirichlet x 64 Fourier, seeded forcing",
            "us_per_solve": us,
            "path": ("one launch (jfb_helmholtz2d_solve: 8-CTA cluster, problem in distributed "
                     "shared memory)" if h.fused else "separate launches"),
            "us_per_solve_graph_replay": us_graph,
            "us_per_solve_separate_launches": us_sep,
            "solves": K,
            "manufactured_rel_l2": err,
            "u_max": float(u.abs().max()),
        }
        if not args.no_cpu_baseline:
            threads = host_threads()
            us_cpu, n = helmholtz_cpu_rate(threads)
            out["cpu_baseline"] = {
                "us_per_solve": us_cpu, "kind": "port", "cores": threads,
                "sample": f"{n} oracle solves, one single-threaded process per core for 2 s "
                          "(throughput over all host cores)"}
        return out

    def default_form_block():
        """The reference's production default on the same workload: the
        gradient nonlinear form u . grad u (FP64) with each time integrator
        the production runner accepts, and its mixed form with SBDF3; ms per
        step (graph replay, CUDA events, L2 not flushed)."""
        out = {}
        f0 = couette_perturbation_fields(grid, domain())
        for integ, prec in (("SBDF3", "fp64"), ("CNAB2", "fp64"), ("IMEXRK222", "fp64"),
                            ("IMEXRK3", "fp64"), ("SBDF3", "mixed")):
            sv = PlaneCouetteFluctuation(N=grid, domain=domain(), Re=RE, dt=DT, device=dev,
                                         time_integrator=integ, nonlinear_form="gradient",
                                         precision=prec)
            e0 = sv.diagnostics(sv.state_from_physical(f0))["Epert"]
            st = sv.solve(sv.state_from_physical(scale_to_energy(f0, e0, ENERGY)), 5)
            torch.cuda.synchronize(dev)
            K = 20
            e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0_.record(stream)
            sv.advance_resident(K)
            e1_.record(stream)
            torch.cuda.synchronize(dev)
            stages = {"SBDF3": 1, "CNAB2": 1, "IMEXRK222": 2, "IMEXRK3": 3}[integ]
            out[integ if prec == "fp64" else f"{integ}_mixed"] = {
                "ms_per_step": e0_.elapsed_time(e1_) / K, "implicit_stages_per_step": stages}
            del sv, st
        out["form"] = ("gradient, FP64 (and SBDF3_mixed: complex64 transforms; tensor-core "
                       "pencil stage where the tiling fits, split periodic transforms with the "
                       "warp-shuffle gradient z stage)")
        return out

    def sizes_block():
        """The same Couette workload at 97^3 and 129^3 (wall-normal points x
        Fourier modes): steady steps/s of both forms (graph replay, CUDA
        events) and the per-field relative L2 distance of the mixed form to
        the FP64 form after 100 and 1000 steps."""
        out = {}
        for n in (97, 129):
            grid_n = (n, n - 1, n - 1)
            f0 = couette_perturbation_fields(grid_n, domain())
            rec = {}
            states = {}
            for prec in ("fp64", "mixed"):
                sv = PlaneCouetteFluctuation(N=grid_n, domain=domain(), Re=RE, dt=DT,
                                             precision=prec, device=dev,
                                             time_integrator="SBDF3", nonlinear_form="rotational")
                if prec == "fp64":
                    e0 = sv.diagnostics(sv.state_from_physical(f0))["Epert"]
                    fields_n = scale_to_energy(f0, e0, ENERGY)
                st = sv.state_from_physical(fields_n)
                tuned = sv.autotune(st, steps=10, cache=False) if not args.no_autotune else None
                st = sv.solve(st, 5)
                torch.cuda.synchronize(dev)
                K = 20
                e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0_.record(stream)
                sv.advance_resident(K)
                e1_.record(stream)
                torch.cuda.synchronize(dev)
                ms = e0_.elapsed_time(e1_) / K
                # per-kernel split (events around each launch, L2 not flushed)
                kms = (ctypes.c_double * 4)()
                sms = ctypes.c_double()
                _lib.call("jfb_kmm_timed_steps", sv._plan, K, None, 0, kms, ctypes.byref(sms),
                          ctypes.c_void_p(stream.cuda_stream))
                torch.cuda.synchronize(dev)
                sv._current = None
                lps = sv.info().launches_per_step
                names = (("pencil_stage", "plane_transforms") if lps == 2 else
                         ("pencil_stage", "y_backward", "z_cross", "y_forward"))
                rec[prec] = {"ms_per_step": ms, "steps_per_s": 1000.0 / ms,
                             "launches_per_step": lps, "autotune": tuned,
                             "kernel_us": {k: kms[i] * 1000.0 / K for i, k in enumerate(names)}}
                states[prec] = (sv, sv.state_from_physical(fields_n))
            (g64, a), (g32, b) = states["fp64"], states["mixed"]
            done = 0
            for m in (100, 1000):
                a, b = g64.solve(a, m - done), g32.solve(b, m - done)
                done = m
                errs = {}
                for name, x, y in zip(("u0", "u1", "u2", "g"), (*b.u, b.g), (*a.u, a.g), strict=True):
                    errs[name] = float(torch.linalg.norm(x - y) / torch.linalg.norm(y))
                num = sum(float(torch.linalg.norm(x - y)) ** 2 for x, y in zip((*b.u, b.g), (*a.u, a.g)))
                den = sum(float(torch.linalg.norm(y)) ** 2 for y in (*a.u, a.g))
                errs["state"] = math.sqrt(num / den)
                rec[f"mixed_vs_fp64_after_{m}_steps"] = errs
            out[f"{n}x{n - 1}x{n - 1}"] = rec
        return out

    def linear_block():
        """Plane-Couette linear stability at Re 1000 on the KMM Legendre
        operators: the leading growth rate of an 8 x 8 (ky, kz) map at nx 64
        (one batched assembly, shift-inverted solve and eigenvalue call), and
        the optimal growth G(t) at 40 times for (ky, kz) = (0, 1.66) at nx 80
        (one batched matrix exponential); CUDA events around each.  CPU
        baseline: the oracle's restatement of the reference's collocation
        operator with QZ, per mode, on the host."""
        import numpy as np

        from jaxfun_b200.linear import PlaneCouetteLinear

        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def timed(fn, reps=3):
            fn()
            torch.cuda.synchronize(dev)
            e0.record(stream)
            for _ in range(reps):
                r = fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            return r, e0.elapsed_time(e1) / reps

        pcf = PlaneCouetteLinear.couette(nx=64, Re=1000.0, device=dev)
        ky, kz = torch.meshgrid(torch.linspace(0.0, 3.0, 8), torch.linspace(0.25, 3.0, 8),
                                indexing="ij")
        rates, ms_map = timed(lambda: pcf.growth_rates(ky, kz), reps=2)
        scan = PlaneCouetteLinear.couette(nx=80, Re=1000.0, device=dev)
        times = np.linspace(120.0, 160.0, 40)
        G, ms_scan = timed(lambda: scan.optimal_growth(0.0, 1.66, times).reshape(-1))
        i = int(G.argmax())
        out = {
            "workload": "plane Couette, Re 1000: leading growth rate over an 8 x 8 (ky, kz) map "
                        "at nx 64; optimal growth at 40 times in [120, 160] for (0, 1.66) at nx 80",
            "growth_rate_map": {"modes": 64, "nx": 64, "ms": ms_map,
                                "max_growth_rate": float(rates.max())},
            "optimal_growth_scan": {"nx": 80, "times": 40, "ms": ms_scan,
                                    "gmax": float(G[i]), "t_opt": float(times[i])},
        }
        if not args.no_cpu_baseline:
            import time as _time

            from oracle.linear import PlaneCouetteLinearOracle
            orc = PlaneCouetteLinearOracle.couette(nx=64, Re=1000.0)
            t0 = _time.perf_counter()
            for kyv, kzv in ((1.0, 1.0), (2.0, 0.5)):
                orc.growth_rate(kyv, kzv)
            per_mode = (_time.perf_counter() - t0) / 2
            orc80 = PlaneCouetteLinearOracle.couette(nx=80, Re=1000.0)
            t0 = _time.perf_counter()
            orc80.nonmodal_growth(0.0, 1.66, times)
            scan_s = _time.perf_counter() - t0
            out["cpu_baseline"] = {
                "kind": "port", "cores": host_threads(),
                "growth_rate_map_ms": per_mode * 64 * 1e3, "optimal_growth_scan_ms": scan_s * 1e3,
                "sample": "2 modes of the map timed and scaled to 64; the full 40-time scan "
                          "(scipy QZ and SVD, default LAPACK threads)"}
        return out

    forms = ("mixed", "fp64") if args.precision == "both" else (args.precision,)
    results = {p: measure(p) for p in forms}
    err = mixed_error() if "mixed" in forms and rank == 0 else None
    adj = adjoint_block() if (rank == 0 and world == 1 and not args.no_adjoint) else None
    ensb = ensemble_block() if (rank == 0 and world == 1 and not args.no_ensemble) else None
    helm = helmholtz_block() if (rank == 0 and world == 1 and not args.no_helmholtz) else None
    lin = linear_block() if (rank == 0 and world == 1 and not args.no_linear) else None
    sizes = sizes_block() if (rank == 0 and world == 1 and not args.no_sizes) else None
    dform = (default_form_block()
             if (rank == 0 and world == 1 and not args.no_default_form) else None)

    if rank != 0:
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return 0

    head = results[forms[0]]
    fields = head.pop("fields")
    line = {
        "metric": METRIC,
        "value": head["value"],
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if forms[0] == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": workload_desc(grid),
        "form": forms[0],
        "l2": "flushed between timed steps (256 MiB memset)",
    }
    line.update({k: v for k, v in head.items() if k not in ("value", "ms_per_step")})
    for p in forms[1:]:
        r = results[p]
        r.pop("fields")
        line[p] = {k: r[k] for k in ("value", "ms_per_step", "roofline", "step_roofline",
                                     "kernel_ms", "graph_l2_resident", "e2e", "gpu_launches",
                                     "autotune")}
    if err is not None:
        line["mixed_vs_fp64_rel_l2"] = err
    if adj is not None:
        line["adjoint"] = adj
        line["adjoint_fd_max_rel_err"] = adj["fd_check"]["max_rel_err"]
    if ensb is not None:
        line["mhd_ensemble"] = ensb
    if helm is not None:
        line["helmholtz2d"] = helm
    if lin is not None:
        line["linear_stability"] = lin
    if sizes is not None:
        line["larger_grids"] = sizes
    if dform is not None:
        line["reference_default_form"] = dform
    if world == 1 and not args.no_cpu_baseline:
        threads = host_threads()
        rate, n = cpu_oracle_rate(fields, grid, args.cpu_seconds, threads)
        line["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n} steady SBDF3 steps of the same workload, oracle restatement, "
                      f"scipy.fft workers={threads}",
        }
    print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
