"""Parity of the CUDA KMM step with the CPU oracle (GPU).

Tolerances: primary fields (u0, u1, u2, g) <= 1e-12 relative L2 (FP64 form);
the nonlinear history rows carry derivative round-off amplification and are
held to 1e-10; diagnostics to 1e-12 relative.
"""

import os

import numpy as np
import pytest
import torch

from jaxfun_b200.kmm import KMMState, PlaneCouetteFluctuation
from oracle.kmm import PlaneCouetteOracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rel(a, b, floor=0.0):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else a
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), floor, 1e-300))


def to_dev(st, dev):
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
    return KMMState(u=tuple(t(a) for a in st.u), g=t(st.g))


def pair(N, Re=600.0, dt=0.01, amp=0.05, dev="cuda"):
    o = PlaneCouetteOracle(N=N, Re=Re, dt=dt, perturbation_amplitude=amp)
    g = PlaneCouetteFluctuation(N=N, Re=Re, dt=dt, perturbation_amplitude=amp, device=dev,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    return o, g


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32), (33, 16, 48)])
def test_convection_matches_oracle(cuda, N):
    o, g = pair(N, dev=cuda)
    st = o.initial_state()
    H = g.convection(to_dev(st, cuda))
    Ho = o.convection(st.u)
    for a, b in zip(H, Ho, strict=True):
        assert rel(a, b) < 1e-12


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32)])
def test_steps_match_oracle(cuda, N):
    o, g = pair(N, Re=400.0, dt=1e-3, dev=cuda)
    st = o.initial_state()
    gs = g._ensure_history(to_dev(st, cuda))
    done = 0
    for n in (1, 2, 3, 8):
        for _ in range(n - done):
            st = o.step(st)
        gs = g.solve(gs, n - done)
        done = n
        for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
            assert rel(a, b) < 1e-12, n
        for lv_g, lv_o in ((gs.solution_old, st.solution_old), (gs.nonlinear_old, st.nonlinear_old)):
            for a, b in zip(lv_g, lv_o, strict=True):
                scale = np.linalg.norm(st.u[1])
                assert rel(a, b, floor=1e-6 * scale) < 1e-10, n
        assert gs.history_steps == min(2.0, float(n))


def test_against_committed_golden_fixture(cuda):
    fx = np.load(os.path.join(HERE, "golden", "pcf_17x16x16.npz"))
    g = PlaneCouetteFluctuation(N=(17, 16, 16), Re=600.0, dt=0.01,
                                perturbation_amplitude=0.05, device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    gs = g.initial_state()
    done = 0
    for n in (0, 3, 10):
        gs = g.solve(gs, n - done) if n > done else gs
        done = n
        for i in range(3):
            assert rel(gs.u[i], fx[f"s{n}_u{i}"]) < 1e-12
        assert rel(gs.g, fx[f"s{n}_g"]) < 1e-12
        d = g.diagnostics(gs)
        names = [str(s) for s in fx["diag_names"]]
        ref = dict(zip(names, fx["diagnostics"][n], strict=True))
        for k in ("Epert", "Etot", "u_top", "u_bot", "wall_shear_top", "mean_shear"):
            assert abs(d[k] - ref[k]) <= 1e-12 * max(1.0, abs(ref[k])), k


def test_initial_state_and_diagnostics_match_oracle(cuda):
    N = (65, 64, 64)
    o, g = pair(N, Re=400.0, dt=1e-3, amp=0.02, dev=cuda)
    st, gs = o.initial_state(), g.initial_state()
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12
    do, dg = o.diagnostics(st), g.diagnostics(gs)
    for k in do:
        if k == "divL2":
            assert abs(dg[k] - do[k]) < 1e-12
        else:
            assert abs(dg[k] - do[k]) <= 1e-12 * max(1.0, abs(do[k])), k


def test_full_size_steps_match_oracle(cuda):
    """65x64x64 (the benchmark grid): startup plus steady steps."""
    N = (65, 64, 64)
    o, g = pair(N, Re=400.0, dt=1e-3, amp=0.02, dev=cuda)
    st, gs = o.initial_state(), g.initial_state()
    st = o.solve(st, 4)
    gs = g.solve(gs, 4)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12


def test_full_size_properties(cuda):
    """Size-independent properties over a longer run at the benchmark grid:
    divergence stays at round-off, the spectrum stays Hermitian, repeated
    runs are bitwise identical, walls keep U = +-1."""
    N = (65, 64, 64)
    g = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    s0 = g.initial_state()
    a = g.solve(s0, 60)
    b = g.solve(s0, 60)
    for x, y in zip((*a.u, a.g), (*b.u, b.g), strict=True):
        assert torch.equal(x, y)
    d = g.diagnostics(a)
    assert d["divL2"] < 1e-12
    assert abs(d["u_top"] - 1.0) < 1e-12 and abs(d["u_bot"] + 1.0) < 1e-12
    assert np.isfinite(d["Epert"]) and d["Epert"] > 0
    u = a.u[1]
    ny, nz = N[1], N[2]
    ky = (-torch.arange(ny, device=u.device)) % ny
    kz = (-torch.arange(nz, device=u.device)) % nz
    mirror = u[:, ky][:, :, kz].conj()
    assert torch.allclose(u, mirror, atol=1e-15 * u.abs().max().item())


def test_solve_rejects_cpu_tensors(cuda):
    g = PlaneCouetteFluctuation(N=(17, 16, 16), device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    st = g.zero_state()
    bad = KMMState(u=tuple(t.cpu() for t in st.u), g=st.g.cpu())
    with pytest.raises(ValueError):
        g.solve(bad, 1)


@pytest.mark.parametrize("N", [(32, 24, 24), (33, 16, 48)])
def test_ragged_tiles_match_oracle(cuda, N):
    """Even Nx (no middle node), Nz/2 not a multiple of 8 (partly empty pencil
    tiles) and Ny != Nz: startup plus steady steps against the oracle."""
    o, g = pair(N, Re=400.0, dt=1e-3, dev=cuda)
    st, gs = o.initial_state(), g.initial_state()
    st = o.solve(st, 5)
    gs = g.solve(gs, 5)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12
    for lv_g, lv_o in ((gs.nonlinear_old, st.nonlinear_old),
                       (gs.nonlinear_older, st.nonlinear_older)):
        for a, b in zip(lv_g, lv_o, strict=True):
            assert rel(a, b, floor=1e-6 * np.linalg.norm(st.u[1])) < 1e-10


@pytest.mark.parametrize("N", [(65, 64, 64), (32, 24, 24)])
def test_tensor_core_and_warp_pencil_kernels_agree(cuda, N, monkeypatch):
    """The tensor-core pencil stage (folded operators) and the warp-per-pencil
    stage (recurrences) are two evaluations of the same step."""
    g1 = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                 device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    monkeypatch.setenv("JFB200_PENCIL", "warp")
    g2 = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                 device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    s0 = g1.initial_state()
    a, b = g1.solve(s0, 12), g2.solve(s0, 12)
    for x, y in zip((*a.u, a.g), (*b.u, b.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-12


@pytest.mark.parametrize("N", [(65, 64, 64), (33, 64, 64)])
def test_fused_and_split_periodic_transforms_agree(cuda, N, monkeypatch):
    """The one-launch plane transforms (CTA pair per x-plane) and the three
    separate transform launches give the same steps."""
    g1 = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                 device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    assert g1.info().launches_per_step == 2
    monkeypatch.setenv("JFB200_TRANSFORMS", "split")
    g2 = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                 device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    assert g2.info().launches_per_step == 4
    s0 = g1.initial_state()
    a, b = g1.solve(s0, 12), g2.solve(s0, 12)
    for x, y in zip((*a.u, a.g), (*b.u, b.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-12


def test_plans_of_different_sizes_and_precisions_coexist(cuda):
    """Building a smaller or mixed-precision plan after a larger one must not
    break the larger plan's launches (kernel attributes are process-wide)."""
    big = PlaneCouetteFluctuation(N=(65, 64, 64), Re=400.0, dt=1e-3, perturbation_amplitude=0.02,
                                  device=cuda,
                                  time_integrator="SBDF3", nonlinear_form="rotational")
    ref = big.solve(big.initial_state(), 3)
    PlaneCouetteFluctuation(N=(33, 32, 32), precision="mixed", device=cuda,
                            time_integrator="SBDF3", nonlinear_form="rotational")
    PlaneCouetteFluctuation(N=(17, 16, 16), device=cuda,
                            time_integrator="SBDF3", nonlinear_form="rotational")
    again = big.solve(big.initial_state(), 3)
    for x, y in zip((*again.u, again.g), (*ref.u, ref.g), strict=True):
        assert torch.equal(x, y)


def _seeded_pair(N, cuda):
    import math

    from jaxfun_b200.workloads import couette_perturbation_fields, scale_to_energy
    dom = ((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi))
    g64 = PlaneCouetteFluctuation(N=N, domain=dom, Re=1000.0, dt=0.01, device=cuda,
                                  time_integrator="SBDF3", nonlinear_form="rotational")
    g32 = PlaneCouetteFluctuation(N=N, domain=dom, Re=1000.0, dt=0.01, precision="mixed",
                                  device=cuda,
                                  time_integrator="SBDF3", nonlinear_form="rotational")
    f = couette_perturbation_fields(N, dom)
    f = scale_to_energy(f, g64.diagnostics(g64.state_from_physical(f))["Epert"], 1e-4)
    return g64, g32, g64.state_from_physical(f), g32.state_from_physical(f)


def test_mixed_form_tracks_fp64(cuda):
    """Mixed form (complex64 transforms of the quadratic product; FP64 Shen
    operators, solves and base-flow terms) against the FP64 form on the seeded
    65x64x64 Couette workload.  Measured: <= 2.2e-9 per field after 100 steps,
    <= 2.5e-8 after 1000."""
    g64, g32, s64, s32 = _seeded_pair((65, 64, 64), cuda)
    for x, y in zip((*s32.u, s32.g), (*s64.u, s64.g), strict=True):
        assert torch.equal(x, y)  # the projection of the initial field is FP64 in both
    done = 0
    for n, tol in ((100, 2e-8), (1000, 2e-7)):
        s64, s32 = g64.solve(s64, n - done), g32.solve(s32, n - done)
        done = n
        for x, y in zip((*s32.u, s32.g), (*s64.u, s64.g), strict=True):
            assert rel(x, y.cpu().numpy()) < tol, n


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32)])
def test_mixed_form_against_oracle(cuda, N):
    o = PlaneCouetteOracle(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05)
    g = PlaneCouetteFluctuation(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05,
                                precision="mixed", device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    st, gs = o.solve(o.initial_state(), 6), g.solve(g.initial_state(), 6)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-7


@pytest.mark.parametrize("N, precision", [((97, 16, 16), "fp64"), ((129, 12, 12), "fp64"),
                                          ((97, 16, 16), "mixed")])
def test_wide_wall_normal_grids_match_oracle(cuda, N, precision):
    """Nx above the tensor-core tiling (97, 129): the warp-per-pencil stage
    with two register rows per lane in its solves, against the oracle.  The
    mixed form is held to its complex64 transform round-off."""
    o = PlaneCouetteOracle(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02)
    g = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                precision=precision, device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    st = o.initial_state()
    gs = g._ensure_history(to_dev(st, cuda))
    for _ in range(4):
        st = o.step(st)
    gs = g.solve(gs, 4)
    tol = 1e-12 if precision == "fp64" else 1e-6
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < tol


@pytest.mark.parametrize("N", [(65, 64, 64), (33, 32, 32)])
def test_tensor_core_velocity_products_track_dmma(cuda, N, monkeypatch):
    """Mixed form with JFB200_TC=1: the velocity / vorticity products of the
    pencil stage on the tcgen05 tensor cores (three-way split-BF16 operands,
    FP32 accumulation in TMEM) against the default FP64 DMMA products.  Both
    round the fields to complex64; the FP32 accumulation leaves the state
    after 12 steps within 5e-8 (measured 1.6e-8 at 65x64x64)."""
    kw = dict(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02, precision="mixed",
              device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    g2 = PlaneCouetteFluctuation(**kw)
    monkeypatch.setenv("JFB200_TC", "1")
    g1 = PlaneCouetteFluctuation(**kw)
    s0 = g1.initial_state()
    a, b = g1.solve(s0, 12), g2.solve(s0, 12)
    for x, y in zip((*a.u, a.g), (*b.u, b.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 5e-8


def test_autotune_selects_a_variant_and_keeps_the_state(cuda, tmp_path, monkeypatch):
    """jfb_kmm_autotune times the plan's kernel variants on copies of the
    loaded state: the state is unchanged afterwards, the chosen variant is
    active and accepted by the plan, and a second call reads the cache."""
    monkeypatch.setenv("JFB200_AUTOTUNE_CACHE", str(tmp_path / "autotune.json"))
    kw = dict(N=(33, 32, 32), Re=1000.0, dt=0.01, perturbation_amplitude=0.02, device=cuda,
              time_integrator="SBDF3", nonlinear_form="rotational")
    ref_solver = PlaneCouetteFluctuation(**kw)
    s0 = ref_solver.initial_state()
    ref = ref_solver.solve(s0, 6)
    g = PlaneCouetteFluctuation(**kw)
    res = g.autotune(s0, steps=5)
    assert res["ms_per_step"] > 0 and not res["cached"]
    assert g.variant()["current"] == res["variant"]
    out = g.solve(s0, 6)  # every variant of the FP64 form agrees to round-off
    for x, y in zip((*out.u, out.g), (*ref.u, ref.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-12
    again = g.autotune(s0, steps=5)
    assert again["cached"] and again["variant"] == res["variant"]
    with pytest.raises(Exception):
        g.set_variant(replicas=99)


@pytest.mark.parametrize("integrator", ["IMEXRK3", "IMEXRK222"])
@pytest.mark.parametrize("N, precision", [((17, 16, 16), "fp64"), ((33, 32, 32), "fp64"),
                                          ((97, 16, 16), "fp64"), ((33, 32, 32), "mixed")])
def test_one_step_integrators_match_oracle(cuda, integrator, N, precision):
    """KMM with time_integrator IMEXRK3 (every step three Spalart stages,
    channelflow_kmm.py:872-935) or IMEXRK222 (two ARS stages,
    channelflow_kmm.py:1137-1192) against the oracle after five steps: FP64
    at 1e-12 on the tensor-core pencil stage (17, 33) and the warp-per-pencil
    stage (97), the mixed form at 1e-7.  The history fields pass through."""
    kw = dict(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05, time_integrator=integrator)
    o = PlaneCouetteOracle(**kw)
    g = PlaneCouetteFluctuation(precision=precision, device=cuda, nonlinear_form="rotational",
                                **kw)
    st = o.initial_state()
    gs = g._ensure_history(to_dev(st, cuda))
    st, gs = o.solve(st, 5), g.solve(gs, 5)
    tol = 1e-12 if precision == "fp64" else 1e-7
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < tol
    assert gs.history_steps == 0.0
    assert all(float(t.abs().max()) == 0.0 for t in gs.nonlinear_old)


def test_set_state_keeps_the_nonnegative_kz_half_of_a_full_complex_state(cuda):
    """Boundary semantics of the half-spectrum storage: a full complex state
    that is not the spectrum of a real field (the reference keeps such states
    as given) is loaded as its kz >= 0 columns; reading it back gives those
    columns unchanged (the Nyquist row ky = -Ny/2 zero, as the reference
    masks it), the kz < 0 columns as the conjugate mirror c(-ky, -kz) =
    conj(c(ky, kz)) and the Nyquist column kz = -Nz/2 zero."""
    g = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=1e-3, device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    rng = np.random.default_rng(7)

    def noise(shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    Nx, Ny, Nz = g.N
    u = (noise((Nx - 4, Ny, Nz)), noise((Nx - 2, Ny, Nz)), noise((Nx - 2, Ny, Nz)))
    gg = noise((Nx - 2, Ny, Nz))
    st = KMMState(u=tuple(torch.from_numpy(a).to(cuda) for a in u),
                  g=torch.from_numpy(gg).to(cuda))
    out = g.solve(st, 0)

    def expected(a):
        e = np.zeros_like(a)
        Kz = Nz // 2
        e[:, :, :Kz] = a[:, :, :Kz]
        e[:, Ny // 2, :Kz] = 0.0
        for kz in range(Kz + 1, Nz):
            for ky in range(Ny):
                e[:, ky, kz] = np.conj(e[:, (Ny - ky) % Ny, Nz - kz])
        return e

    assert np.array_equal(out.u[0].cpu().numpy(), expected(u[0]))
    assert np.array_equal(out.g.cpu().numpy(), expected(gg))
