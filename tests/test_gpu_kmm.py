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
    g = PlaneCouetteFluctuation(N=N, Re=Re, dt=dt, perturbation_amplitude=amp, device=dev)
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
                                perturbation_amplitude=0.05, device=cuda)
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
                                device=cuda)
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
    g = PlaneCouetteFluctuation(N=(17, 16, 16), device=cuda)
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
                                 device=cuda)
    monkeypatch.setenv("JFB200_PENCIL", "warp")
    g2 = PlaneCouetteFluctuation(N=N, Re=1000.0, dt=0.01, perturbation_amplitude=0.02,
                                 device=cuda)
    s0 = g1.initial_state()
    a, b = g1.solve(s0, 12), g2.solve(s0, 12)
    for x, y in zip((*a.u, a.g), (*b.u, b.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-12
