"""Phase split of the two step kernels from the phase-stamp build.

Usage (profiling only; needs ``libjfb200_stamps.so``, built by
``python -m jaxfun_b200.build --stamps``)::

    JFB200_LIB=jaxfun_b200/libjfb200_stamps.so python -m jaxfun_b200.phase_stamps \\
        --precision mixed --grid 65,64,64

Runs the benchmark workload (seeded Couette perturbation, Re 1000, dt 0.01)
for a few steps, then one steady step after a 256 MiB L2 flush, and prints
per-phase durations of ``pencil_gemm_kernel`` (kernel 0) and
``plane_cross_kernel`` (kernel 1): the median over CTAs of each interval
between consecutive stamps, and the median CTA's total.  Phase names follow
the stamp points in the kernels (jfb_kmm_gemm.cuh, jfb_kmm_warpk.cuh).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import math
import statistics

PENCIL = ("launch+prologue", "staging", "mirror+mass inputs", "B products", "C1 elimination",
          "C2 U^-1 products", "C3 stores+wait", "D velocity", "middle node")
PLANE = ("launch+wait", "y staging", "y inverse FFT", "z stage", "y forward FFT",
         "stores", "cluster exit")


def main(argv=None) -> int:
    import torch

    from . import _lib
    from .kmm import PlaneCouetteFluctuation
    from .workloads import couette_perturbation_fields, scale_to_energy

    p = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    p.add_argument("--precision", default="mixed", choices=("mixed", "fp64"))
    p.add_argument("--grid", default="65,64,64")
    p.add_argument("--repeats", type=int, default=5)
    a = p.parse_args(argv)
    lib = _lib.load()
    if not hasattr(lib, "jfb_debug_read_stamps"):
        raise SystemExit("load the stamp build: JFB200_LIB=.../libjfb200_stamps.so")
    lib.jfb_debug_read_stamps.argtypes = [ctypes.c_void_p, ctypes.c_int64]
    grid = tuple(int(v) for v in a.grid.split(","))
    dom = ((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi))
    dev = torch.device("cuda", 0)
    g = PlaneCouetteFluctuation(N=grid, domain=dom, Re=1000.0, dt=0.01, precision=a.precision,
                                device=dev, time_integrator="SBDF3", nonlinear_form="rotational")
    f = couette_perturbation_fields(grid, dom)
    f = scale_to_energy(f, g.diagnostics(g.state_from_physical(f))["Epert"], 1e-4)
    g.solve(g.state_from_physical(f), 5)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    n_cta, n_ph = 1024, 16
    out = {"grid": list(grid), "precision": a.precision, "unit": "us"}
    runs = {0: [], 1: []}
    for _ in range(a.repeats):
        flush.fill_(1)
        g.advance_resident(1)
        torch.cuda.synchronize(dev)
        buf = (ctypes.c_ulonglong * (4 * n_cta * n_ph))()
        _lib.check(lib.jfb_debug_read_stamps(buf, 4 * n_cta * n_ph))
        for k, nph in ((0, len(PENCIL) + 1), (1, len(PLANE) + 1)):
            ctas = []
            for c in range(n_cta):
                st = [buf[(k * n_cta + c) * n_ph + i] for i in range(nph)]
                if all(st) and all(st[i + 1] >= st[i] for i in range(nph - 1)):
                    ctas.append(st)
            runs[k].append(ctas)
    for k, names in ((0, PENCIL), (1, PLANE)):
        last = runs[k][-1]
        if not last:
            continue
        t0 = min(c[0] for c in last)
        per = {n: statistics.median(
            statistics.median((c[i + 1] - c[i]) / 1e3 for c in r) for r in runs[k] if r)
            for i, n in enumerate(names)}
        tot = statistics.median(statistics.median((c[-1] - c[0]) / 1e3 for c in r)
                                for r in runs[k] if r)
        span = (max(c[-1] for c in last) - t0) / 1e3
        rec = {"ctas": len(last), "phases_median_cta": per, "cta_total_median": tot,
               "first_start_to_last_end": span}
        if k == 0:  # tensor-core velocity stage (JFB200_TC=1): stamps 10-13 inside D
            sub = []
            for c in range(n_cta):
                st = [buf[c * n_ph + i] for i in (7, 10, 11, 12, 13, 8)]
                if all(st) and all(st[i + 1] >= st[i] for i in range(5)):
                    sub.append(st)
            if sub:
                names = ("D: state split", "D: MMA issue", "D: MMA wait", "D: TMEM load",
                         "D: epilogue")
                rec["tc_subphases_median_cta"] = {
                    n: statistics.median((c[i + 1] - c[i]) / 1e3 for c in sub)
                    for i, n in enumerate(names)}
        out["pencil_gemm" if k == 0 else "plane_cross"] = rec
    print(json.dumps(out))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
