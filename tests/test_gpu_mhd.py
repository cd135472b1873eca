"""Parity of the CUDA plane-Couette MHD step with the CPU oracle (GPU).

Tolerances (FP64): flow fields and A <= 1e-12 relative L2 (components that
start at zero are measured against the norm of A as a whole); the EMF
history rows <= 1e-10; nonlinear terms <= 1e-12; diagnostics <= 1e-12
relative, divB_L2 at round-off.
"""

import numpy as np
import pytest
import torch

from jaxfun_b200.kmm import KMMState
from jaxfun_b200.mhd import MHDState, PlaneCouetteMHD
from oracle.kmm import PlaneCouetteMHDOracle

pytestmark = pytest.mark.gpu


def rel(a, b, floor=0.0):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else a
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), floor, 1e-300))


def t(a, dev):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


def to_dev(st, dev):
    flow = KMMState(u=tuple(t(a, dev) for a in st.flow.u), g=t(st.flow.g, dev))
    return MHDState(flow=flow, A=tuple(t(a, dev) for a in st.A))


def pair(N, dev, Re=400.0, Rm=None, dt=1e-3, amp=0.05, mag=0.05):
    kw = dict(N=N, Re=Re, Rm=Rm, dt=dt, perturbation_amplitude=amp, magnetic_amplitude=mag)
    return PlaneCouetteMHDOracle(**kw), PlaneCouetteMHD(device=dev, **kw)


def a_scale(A):
    return max(np.linalg.norm(a) for a in A)


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32)])
def test_initial_potential_matches_oracle(cuda, N):
    o, g = pair(N, cuda)
    st, gs = o.initial_state(), g.initial_state()
    for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
        assert rel(a, b) < 1e-12
    sc = a_scale(st.A)
    for a, b in zip(gs.A, st.A, strict=True):
        assert rel(a, b, floor=sc) < 1e-13
    assert gs.flow.history_steps == 0.0


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 48)])
def test_convection_matches_oracle(cuda, N):
    """H = TD[-(u_t x w_t) - J x B] and HA = TD[(u + U_b) x B] of one state."""
    o, g = pair(N, cuda, amp=0.05, mag=0.2)
    st = o.initial_state()
    # a state with all three A components and a richer flow: two oracle steps
    st = o.solve(st, 2)
    H, HA = g.convection(to_dev(st, cuda))
    Ho, HAo = o.mhd_convection(st)
    for a, b in zip(H, Ho, strict=True):
        assert rel(a, b) < 1e-12
    sc = max(np.linalg.norm(h) for h in HAo)
    for a, b in zip(HA, HAo, strict=True):
        assert rel(a, b, floor=sc) < 1e-12


@pytest.mark.parametrize("N, Rm", [((17, 16, 16), None), ((33, 32, 32), 150.0)])
def test_steps_match_oracle(cuda, N, Rm):
    """IMEXRK3 startup steps, then steady SBDF3 steps; eta != nu when Rm != Re."""
    o, g = pair(N, cuda, Rm=Rm, mag=0.2)
    st, gs = o.initial_state(), g.initial_state()
    done = 0
    for n in (1, 2, 3, 8):
        st = o.solve(st, n - done)
        gs = g.solve(gs, n - done)
        done = n
        for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
            assert rel(a, b) < 1e-12, n
        sc = a_scale(st.A)
        for a, b in zip(gs.A, st.A, strict=True):
            assert rel(a, b, floor=sc) < 1e-12, n
        for a, b in zip(gs.A_old, st.A_old, strict=True):
            assert rel(a, b, floor=sc) < 1e-12, n
        sn = a_scale(st.nonlinear_A_old)
        for a, b in zip(gs.nonlinear_A_old, st.nonlinear_A_old, strict=True):
            assert rel(a, b, floor=sn) < 1e-10, n
        assert gs.flow.history_steps == min(2.0, float(n))


def test_diagnostics_match_oracle(cuda):
    o, g = pair((33, 32, 32), cuda, mag=0.2)
    st, gs = o.solve(o.initial_state(), 3), g.solve(g.initial_state(), 3)
    do, dg = o.diagnostics(st), g.diagnostics(gs)
    assert set(do) == set(dg)
    for k in do:
        if k in ("divL2", "divB_L2"):
            assert dg[k] < 1e-13 and do[k] < 1e-13, k
        else:
            assert abs(dg[k] - do[k]) <= 1e-12 * max(1.0, abs(do[k])), k
    assert dg["Emag"] > 0


def test_state_round_trip_continues_identically(cuda):
    """get_state / set_state of the full MHDState (history included) loses
    nothing: continuing from a reloaded state equals continuing in place up to
    the round-off of recomputing the loaded state's nonlinear terms (the
    in-place path reuses those of the step that produced it)."""
    g = PlaneCouetteMHD(N=(17, 16, 16), dt=1e-3, magnetic_amplitude=0.2, device=cuda)
    s = g.solve(g.initial_state(), 4)
    a = g.solve(s, 3)
    g._current = None
    b = g.solve(s, 3)
    sc = a_scale([x.cpu().numpy() for x in a.A])
    for x, y in zip((*a.flow.u, a.flow.g), (*b.flow.u, b.flow.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-13
    for x, y in zip(a.A, b.A, strict=True):
        assert rel(x, y.cpu().numpy(), floor=sc) < 1e-13


def test_benchmark_grid_properties(cuda):
    """65x64x64: startup plus steady steps against the oracle, then
    divergence-free B and a finite, positive magnetic energy."""
    N = (65, 64, 64)
    o, g = pair(N, cuda, amp=0.02, mag=0.005)
    st, gs = o.solve(o.initial_state(), 4), g.solve(g.initial_state(), 4)
    for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
        assert rel(a, b) < 1e-12
    sc = a_scale(st.A)
    for a, b in zip(gs.A, st.A, strict=True):
        assert rel(a, b, floor=sc) < 1e-12
    d = g.diagnostics(gs)
    assert d["divB_L2"] < 1e-14 and d["Emag"] > 0


def test_mhd_plan_rejects_flow_states(cuda):
    g = PlaneCouetteMHD(N=(17, 16, 16), device=cuda)
    flow = g.initial_state().flow
    with pytest.raises(TypeError):
        g.solve(flow, 1)


def test_initial_magnetic_energy_is_analytic(cuda):
    """Emag of the seed potential (exact, see the oracle unit test)."""
    a = 0.2
    g = PlaneCouetteMHD(N=(33, 32, 32), dt=1e-3, magnetic_amplitude=a, device=cuda)
    d = g.diagnostics(g.initial_state())
    Ly, Lz = 4.0 * np.pi, 2.0 * np.pi
    exact = a * a * (16.0 / 15.0) * (Ly * Lz / 4.0) * (1.0 + (Lz / Ly) ** 2)
    assert abs(d["Emag"] - exact) < 1e-13 * exact
    assert d["divB_L2"] < 1e-15


def test_reference_mhd_benchmark_golden(cuda):
    """The reference's recorded MHD benchmark (65x64x64, Re = Rm = 400,
    dt = 1e-3, 325 SBDF3 rotational steps): final diagnostics to 1e-10."""
    import json
    import os

    spec = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                       "reference_goldens.json")))
    spec = spec["benchmark_mhd_sbdf3_rotational_65x64x64"]
    s = spec["solver"]
    g = PlaneCouetteMHD(N=tuple(s["N"]), Re=s["Re"], Rm=s["Rm"], dt=s["dt"],
                        perturbation_amplitude=s["perturbation_amplitude"],
                        magnetic_amplitude=s["magnetic_amplitude"], device=cuda)
    d = g.diagnostics(g.solve(g.initial_state(), spec["steps"]))
    for key in ("Emag", "Epert", "Etot", "wall_shear_top", "wall_shear_bot", "u_top", "u_bot"):
        ref = spec["diagnostics"][key]
        assert abs(d[key] - ref) <= 1e-10 * abs(ref) + 1e-14, key
    assert d["divB_L2"] < 1e-15 and d["divL2"] < 1e-15


def test_rotating_shear_variant_matches_oracle(cuda):
    """PlaneCouetteMRIShearpyJax dynamics: U_b = -S x, Coriolis, imposed B0,
    eta = 1/Rm != nu (pcf_mhd_mri_shearpy_jax.py:36-176)."""
    from jaxfun_b200.mhd import PlaneCouetteMRIShearpy
    from oracle.kmm import PlaneCouetteMRIOracle

    kw = dict(N=(17, 16, 16), Re=400.0, Rm=250.0, omega=0.5, shear_rate=1.5,
              background_b=(0.01, 0.02, 0.1), dt=1e-3, magnetic_amplitude=0.2)
    o = PlaneCouetteMRIOracle(**kw)
    g = PlaneCouetteMRIShearpy(device=cuda, **kw)
    st = o.initial_state()
    gs = to_dev(st, cuda)
    done = 0
    for n in (1, 2, 3, 6):
        st = o.solve(st, n - done)
        gs = g.solve(gs, n - done)
        done = n
        for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
            assert rel(a, b) < 1e-12, n
        sc = a_scale(st.A)
        for a, b in zip(gs.A, st.A, strict=True):
            assert rel(a, b, floor=sc) < 1e-12, n
    do, dg = o.diagnostics(st), g.diagnostics(gs)
    for k in ("Epert", "Etot", "u_top", "u_bot", "wall_shear_top", "Emag"):
        assert abs(dg[k] - do[k]) <= 1e-12 * max(1.0, abs(do[k])), k


@pytest.mark.parametrize("precision, tol", [("fp64", 1e-12), ("mixed", 5e-6)])
def test_rotating_shear_convection_matches_oracle(cuda, precision, tol):
    """H and HA of a rotating-shear state with an imposed field (the EMF's
    U_b e_y x B0 term reaches only the mean mode, which the A stage adds in
    FP64)."""
    from jaxfun_b200.mhd import PlaneCouetteMRIShearpy
    from oracle.kmm import PlaneCouetteMRIOracle

    kw = dict(N=(17, 16, 16), Re=400.0, Rm=250.0, omega=0.5, shear_rate=1.5,
              background_b=(0.01, 0.02, 0.1), dt=1e-3, magnetic_amplitude=0.2)
    o = PlaneCouetteMRIOracle(**kw)
    g = PlaneCouetteMRIShearpy(device=cuda, precision=precision, **kw)
    st = o.solve(o.initial_state(), 2)
    H, HA = g.convection(to_dev(st, cuda))
    Ho, HAo = o.mhd_convection(st)
    for a, b in zip(H, Ho, strict=True):
        assert rel(a, b) < tol
    sc = max(np.linalg.norm(h) for h in HAo)
    for a, b in zip(HA, HAo, strict=True):
        assert rel(a, b, floor=sc) < tol


def test_ensemble_of_uneven_members_equals_separate_runs(cuda):
    """Members of uneven wall-normal size (and a flow-only member) advanced
    as one graph per step give bitwise the results of separate runs."""
    from jaxfun_b200.kmm import PlaneCouetteFluctuation
    from jaxfun_b200.mhd import Ensemble

    def members():
        return [PlaneCouetteMHD(N=(17, 16, 16), dt=1e-3, magnetic_amplitude=0.1, device=cuda),
                PlaneCouetteMHD(N=(25, 16, 16), dt=1e-3, magnetic_amplitude=0.1, device=cuda),
                PlaneCouetteMHD(N=(33, 16, 16), dt=1e-3, magnetic_amplitude=0.1, device=cuda),
                PlaneCouetteFluctuation(N=(33, 16, 16), dt=1e-3, device=cuda,
                                        time_integrator="SBDF3", nonlinear_form="rotational")]

    sep = members()
    ref = [m.solve(m.initial_state(), 7) for m in sep]
    ens_m = members()
    ens = Ensemble(ens_m)
    out = ens.solve([m.initial_state() for m in ens_m], 7)
    for a, b in zip(out, ref, strict=True):
        if isinstance(a, MHDState):
            la, lb = (*a.flow.u, a.flow.g, *a.A), (*b.flow.u, b.flow.g, *b.A)
        else:
            la, lb = (*a.u, a.g), (*b.u, b.g)
        for x, y in zip(la, lb, strict=True):
            assert torch.equal(x, y)


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32), (65, 64, 64)])
def test_mixed_form_tracks_the_oracle(cuda, N):
    """Mixed MHD form: complex64 periodic transforms and products of u,
    omega, b, j (the flow's base-flow terms added in FP64 by the pencil
    stage), FP64 operators, solves and state.  Against the FP64 oracle after
    two startup and six steady steps: every field within 5e-8 relative L2
    (measured <= 1.1e-8)."""
    kw = dict(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05, magnetic_amplitude=0.2)
    o = PlaneCouetteMHDOracle(**kw)
    g = PlaneCouetteMHD(device=cuda, precision="mixed", **kw)
    st = o.initial_state()
    gs = g.solve(to_dev(st, cuda), 8)
    st = o.solve(st, 8)
    for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
        assert rel(a, b) < 5e-8
    sc = a_scale(st.A)
    for a, b in zip(gs.A, st.A, strict=True):
        assert rel(a, b, floor=sc) < 5e-8


def test_mixed_rotating_shear_variant_tracks_the_oracle(cuda):
    """The rotating-shear variant (imposed B0, Coriolis, eta != nu) in the
    mixed form: within 2e-8 of the oracle after six steps (measured 5e-9)."""
    from jaxfun_b200.mhd import PlaneCouetteMRIShearpy
    from oracle.kmm import PlaneCouetteMRIOracle

    kw = dict(N=(33, 32, 32), Re=400.0, Rm=250.0, omega=0.5, shear_rate=1.5,
              background_b=(0.01, 0.02, 0.1), dt=1e-3, magnetic_amplitude=0.2)
    o = PlaneCouetteMRIOracle(**kw)
    g = PlaneCouetteMRIShearpy(device=cuda, precision="mixed", **kw)
    st = o.initial_state()
    gs = g.solve(to_dev(st, cuda), 6)
    st = o.solve(st, 6)
    for a, b in zip((*gs.flow.u, gs.flow.g), (*st.flow.u, st.flow.g), strict=True):
        assert rel(a, b) < 2e-8
    sc = a_scale(st.A)
    for a, b in zip(gs.A, st.A, strict=True):
        assert rel(a, b, floor=sc) < 2e-8


def test_mixed_batched_ensemble_equals_separate_runs(cuda):
    """Mixed-form members of uneven wall-normal size: the batched stages
    (complex64 transform stages) give each member bitwise its own plan's
    result."""
    from jaxfun_b200.mhd import Ensemble

    def members():
        return [PlaneCouetteMHD(N=(n, 64, 64), dt=1e-3, magnetic_amplitude=0.1,
                                precision="mixed", device=cuda) for n in (33, 17, 25, 33)]

    ref = [m.solve(m.initial_state(), 7) for m in members()]
    ms = members()
    ens = Ensemble(ms)
    assert ens.batched and ens.launches_per_step == 15
    out = ens.solve([m.initial_state() for m in ms], 7)
    for a, b in zip(out, ref, strict=True):
        for x, y in zip((*a.flow.u, a.flow.g, *a.A), (*b.flow.u, b.flow.g, *b.A), strict=True):
            assert torch.equal(x, y)


def test_batched_ensemble_of_uneven_mhd_members_equals_separate_runs(cuda, monkeypatch):
    """All-MHD ensembles of uneven wall-normal size advance as five launches
    per steady step for each wall-normal size (one per stage, a work list
    over that size's members' tiles, the sizes on parallel graph branches),
    or as five launches over all members (JFB200_ENSEMBLE=batched); either
    result is bitwise that of separate runs, and that of the
    one-stream-per-member graph (five launches per member)."""
    from jaxfun_b200.mhd import Ensemble

    def members():
        # 64 Fourier modes: padded length 96 = 32 x 3, the warp-FFT y transforms
        return [PlaneCouetteMHD(N=(n, 64, 64), dt=1e-3, magnetic_amplitude=0.1, device=cuda)
                for n in (33, 17, 25, 33)]

    sep = members()
    ref = [m.solve(m.initial_state(), 7) for m in sep]
    outs = []
    for mode, batched, launches in ((None, True, 15), ("batched", True, 5),
                                    ("streams", False, 20)):
        if mode is None:
            monkeypatch.delenv("JFB200_ENSEMBLE", raising=False)
        else:
            monkeypatch.setenv("JFB200_ENSEMBLE", mode)
        ms = members()
        ens = Ensemble(ms)
        assert ens.batched == batched, mode
        assert ens.launches_per_step == launches, mode
        outs.append(ens.solve([m.initial_state() for m in ms], 7))
    for a, b, c, d in zip(*outs, ref, strict=True):
        la, lb, lc, ld = ((*x.flow.u, x.flow.g, *x.A) for x in (a, b, c, d))
        for x, y, z, w in zip(la, lb, lc, ld, strict=True):
            assert torch.equal(x, w) and torch.equal(y, w) and torch.equal(z, w)
