"""Parity of the CUDA step on the configurations the benchmark measures (GPU).

* The reference's own recorded hydro benchmark (65x64x64, Re 400, dt 1e-3,
  amplitude 0.02, 325 SBDF3 rotational steps,
  benchmark-results/hydro-sbdf3-rotational-65x64x64-r2.json): final
  diagnostics to 1e-10 and the full-state L2 checksum over the state tree
  (u, g and both history levels) with its element count.
* The benchmark workload itself (65x64x64, Re 1000, dt 0.01, the seeded
  divergence-free perturbation of ``jaxfun_b200.workloads`` at energy 1e-4):
  FP64 against the oracle after 100 steps at 1e-12 per field, the mixed form
  at 2e-8 (its complex64 transform round-off; measured about 2e-9).
* The larger grids of the mixed-precision configuration (97x96x96 and
  129x128x128), both forms against the oracle after two IMEXRK3 startup
  steps and one steady SBDF3 step of the analytic field: FP64 at 1e-12,
  mixed at 2e-7 (measured 3.9e-8 / 5.5e-8: the modes this field excites
  only through the nonlinear term are ~1e-9 in size, and the complex64
  transforms resolve them to FP32 round-off of the O(1) fields).
* A state with a NaN injected on the host raises ``FloatingPointError``
  after the step, and the plan keeps working afterwards.
"""

import json
import math
import os
from dataclasses import replace

import numpy as np
import pytest
import torch

from jaxfun_b200.kmm import KMMState, PlaneCouetteFluctuation
from jaxfun_b200.workloads import couette_perturbation_fields, scale_to_energy
from oracle.kmm import PlaneCouetteOracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
DOMAIN = ((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi))


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else a
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def to_dev(st, dev):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    return KMMState(u=tuple(t(a) for a in st.u), g=t(st.g))


def test_reference_hydro_benchmark_golden_on_gpu(cuda):
    spec = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))
    spec = spec["benchmark_hydro_sbdf3_rotational_65x64x64"]
    s = spec["solver"]
    g = PlaneCouetteFluctuation(N=tuple(s["N"]), Re=s["Re"], dt=s["dt"],
                                perturbation_amplitude=s["perturbation_amplitude"],
                                padding_factor=tuple(s["padding_factor"]), device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    st = g.solve(g.initial_state(), spec["steps"])
    d = g.diagnostics(st)
    for key in ("Epert", "Etot", "wall_shear_top", "wall_shear_bot", "u_top", "u_bot",
                "mean_shear"):
        ref = spec["diagnostics"][key]
        assert abs(d[key] - ref) <= 1e-10 * abs(ref) + 1e-14, key
    assert d["divL2"] < 1e-15
    # the reference's state checksum: every leaf of the state tree plus the
    # three scalars (history_steps = 2, step counter 1, dt)
    leaves = (list(st.u) + [st.g] + list(st.nonlinear_old) + list(st.nonlinear_older)
              + list(st.solution_old) + list(st.solution_older))
    count = sum(a.numel() for a in leaves) + 3
    sq = sum(float(torch.sum(a.abs() ** 2)) for a in leaves)
    l2 = math.sqrt(sq + 4.0 + 1.0 + s["dt"] ** 2)
    cs = spec["state_checksum"]
    assert count == cs["element_count"]
    assert abs(l2 - cs["l2_norm"]) <= 1e-10 * cs["l2_norm"]


@pytest.fixture(scope="module")
def bench_workload(cuda):
    """The benchmark's seeded 65x64x64 field, projected by the GPU and by the
    oracle from the same physical samples."""
    N = (65, 64, 64)
    g64 = PlaneCouetteFluctuation(N=N, domain=DOMAIN, Re=1000.0, dt=0.01, device=cuda,
                                  time_integrator="SBDF3", nonlinear_form="rotational")
    g32 = PlaneCouetteFluctuation(N=N, domain=DOMAIN, Re=1000.0, dt=0.01, precision="mixed",
                                  device=cuda,
                                  time_integrator="SBDF3", nonlinear_form="rotational")
    o = PlaneCouetteOracle(N=N, domain=DOMAIN, Re=1000.0, dt=0.01)
    f = couette_perturbation_fields(N, DOMAIN)
    f = scale_to_energy(f, g64.diagnostics(g64.state_from_physical(f))["Epert"], 1e-4)
    s_gpu = g64.state_from_physical(f)
    s_orc = o.state_from_physical(tuple(np.asarray(v, dtype=complex) for v in f))
    return g64, g32, o, s_gpu, s_orc


def test_bench_workload_initial_state_matches_oracle(bench_workload):
    g64, _, o, s_gpu, s_orc = bench_workload
    for a, b in zip((*s_gpu.u, s_gpu.g), (*s_orc.u, s_orc.g), strict=True):
        assert rel(a, b) < 1e-12
    assert abs(g64.diagnostics(s_gpu)["Epert"] - 1e-4) < 1e-16


def test_bench_workload_100_steps_both_forms_against_oracle(bench_workload):
    g64, g32, o, s_gpu, s_orc = bench_workload
    ref = o.solve(s_orc, 100)
    a = g64.solve(s_gpu, 100)
    b = g32.solve(s_gpu, 100)
    for x, y in zip((*a.u, a.g), (*ref.u, ref.g), strict=True):
        assert rel(x, y) < 1e-12
    for x, y in zip((*b.u, b.g), (*ref.u, ref.g), strict=True):
        assert rel(x, y) < 2e-8
    do, dg = o.diagnostics(ref), g64.diagnostics(a)
    for k in ("Epert", "Etot", "wall_shear_top", "wall_shear_bot"):
        assert abs(dg[k] - do[k]) <= 1e-12 * abs(do[k]), k


@pytest.mark.parametrize("N", [(97, 96, 96), (129, 128, 128)])
def test_large_grids_both_forms_against_oracle(cuda, N):
    o = PlaneCouetteOracle(N=N, domain=DOMAIN, Re=1000.0, dt=0.01,
                           perturbation_amplitude=0.02)
    st = o.initial_state()
    ref = o.solve(st, 3)  # two IMEXRK3 startup steps, one steady SBDF3 step
    for precision, tol in (("fp64", 1e-12), ("mixed", 2e-7)):
        g = PlaneCouetteFluctuation(N=N, domain=DOMAIN, Re=1000.0, dt=0.01,
                                    perturbation_amplitude=0.02, precision=precision,
                                    device=cuda,
                                    time_integrator="SBDF3", nonlinear_form="rotational")
        gs = g.solve(g._ensure_history(to_dev(st, cuda)), 3)
        for x, y in zip((*gs.u, gs.g), (*ref.u, ref.g), strict=True):
            assert rel(x, y) < tol, precision
        del g


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_nonfinite_state_raises_floating_point_error(cuda, precision):
    """A NaN injected on the host into the loaded state: the step's status word
    reports it and ``solve`` raises FloatingPointError (the reference's runner
    raises it for a non-finite state, production/oracles.py:3257-3261)."""
    g = PlaneCouetteFluctuation(N=(33, 32, 32), Re=400.0, dt=1e-3, precision=precision,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    st = g.initial_state()
    u0 = st.u[0].cpu()
    u0[5, 3, 2] = complex(float("nan"), 0.0)
    bad = replace(st, u=(u0.to(cuda), st.u[1], st.u[2]))
    with pytest.raises(FloatingPointError):
        g.solve(bad, 2)
    # the word was cleared: a finite state advances normally afterwards
    good = g.solve(st, 2)
    assert all(bool(torch.isfinite(torch.view_as_real(t)).all()) for t in (*good.u, good.g))
    g.check()
