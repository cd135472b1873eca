"""The Legendre family and the gradient nonlinear form on the GPU step.

The reference's default solver (examples/pcf_fluctuations_jax.py:35-75) is
the gradient form u . grad u with the IMEXRK222 integrator; its recorded
one-step golden (tests/couette/test_pcf_fluctuations_jax.py:218-238) is a
Legendre run.  Tolerances: the golden's own (rtol 1e-10, atol 1e-12; divL2
atol 5e-15); GPU against the FP64 oracle 1e-12 relative L2 on the primary
fields (u0, u1, u2, g), 1e-10 on the history rows.
"""

import json
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


def test_reference_one_step_legendre_golden_on_gpu(cuda):
    """The reference's recorded diagnostics after one IMEXRK222 step of the
    Legendre (9, 8, 8) gradient-form solver with its default arguments."""
    with open(os.path.join(HERE, "golden", "reference_goldens.json")) as f:
        gold = json.load(f)["one_step_legendre_9x8x8"]
    sv = gold["solver"]
    g = PlaneCouetteFluctuation(N=tuple(sv["N"]), family="L", dt=sv["dt"],
                                perturbation_amplitude=sv["perturbation_amplitude"],
                                device=cuda)
    assert g.time_integrator == "IMEXRK222" and g.nonlinear_form == "gradient"
    st = g.step(g.initial_state())
    d = g.diagnostics(st)
    for key, value in gold["diagnostics"].items():
        atol = 1.0e-12 if key != "divL2" else 5.0e-15
        assert abs(d[key] - value) <= atol + gold["rtol"] * abs(value), (key, d[key], value)


CASES = [
    # (N, family, form, integrator, Re, dt)
    ((17, 16, 16), "C", "gradient", "SBDF3", 400.0, 1e-3),
    ((17, 16, 16), "L", "gradient", "SBDF3", 400.0, 1e-3),
    ((17, 16, 16), "L", "rotational", "SBDF3", 400.0, 1e-3),
    ((9, 8, 8), "L", "gradient", "IMEXRK222", 600.0, 1e-3),
    ((17, 16, 16), "C", "gradient", "IMEXRK3", 400.0, 1e-3),
    ((33, 32, 32), "C", "gradient", "SBDF3", 400.0, 1e-3),
    ((33, 16, 48), "L", "gradient", "SBDF3", 400.0, 1e-3),
    ((17, 16, 16), "C", "gradient", "CNAB2", 400.0, 1e-3),
    ((17, 16, 16), "L", "rotational", "CNAB2", 400.0, 1e-3),
    ((33, 32, 32), "C", "rotational", "CNAB2", 400.0, 1e-3),
]


@pytest.mark.parametrize("N,family,form,integrator,Re,dt", CASES)
def test_forms_match_oracle(cuda, N, family, form, integrator, Re, dt):
    kw = dict(family=family, nonlinear_form=form, time_integrator=integrator)
    o = PlaneCouetteOracle(N=N, Re=Re, dt=dt, perturbation_amplitude=0.05, **kw)
    g = PlaneCouetteFluctuation(N=N, Re=Re, dt=dt, perturbation_amplitude=0.05,
                                device=cuda, **kw)
    st = o.initial_state()
    gs0 = g.initial_state()
    for a, b in zip((*gs0.u, gs0.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12
    H = g.convection(gs0)
    for a, b in zip(H, o.convection(st.u), strict=True):
        assert rel(a, b) < 1e-12
    gs = g._ensure_history(to_dev(st, cuda))
    done = 0
    for n in (1, 2, 4):
        for _ in range(n - done):
            st = o.step(st)
        gs = g.solve(gs, n - done)
        done = n
        for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
            assert rel(a, b) < 1e-12, n
        levels = {"SBDF3": ("solution_old", "nonlinear_old"), "CNAB2": ("nonlinear_old",)}
        for name in levels.get(integrator, ()):
            for a, b in zip(getattr(gs, name), getattr(st, name), strict=True):
                scale = np.linalg.norm(st.u[1])
                assert rel(a, b, floor=1e-6 * scale) < 1e-10, (n, name)
        if integrator == "CNAB2":
            assert gs.have_old == 1.0 and gs.previous_dt == dt
    do, dg = o.diagnostics(st), g.diagnostics(gs)
    for k in do:
        tol = 1e-12 * max(1.0, abs(do[k]))
        assert abs(dg[k] - do[k]) <= tol, (k, dg[k], do[k])


def test_gradient_form_full_size_warp_transforms(cuda):
    """65 x 64 x 64: the gradient form's y transforms on the warp-shuffle
    path (96 = 32 x 3), startup and a steady step against the oracle."""
    N = (65, 64, 64)
    kw = dict(nonlinear_form="gradient", time_integrator="SBDF3")
    o = PlaneCouetteOracle(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.02, **kw)
    g = PlaneCouetteFluctuation(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.02,
                                device=cuda, **kw)
    st = o.initial_state()
    gs = g._ensure_history(to_dev(st, cuda))
    for _ in range(4):
        st = o.step(st)
    gs = g.solve(gs, 4)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12


def test_legendre_tensor_core_and_warp_pencil_stages_agree(cuda):
    """Legendre rotational form at 33^3 on both pencil kernels."""
    N = (33, 32, 32)
    kw = dict(family="L", nonlinear_form="rotational", time_integrator="SBDF3")
    a = PlaneCouetteFluctuation(N=N, Re=400.0, dt=1e-3, device=cuda, **kw)
    b = PlaneCouetteFluctuation(N=N, Re=400.0, dt=1e-3, device=cuda, **kw)
    if not a.variant()["available"]["pencil"]:
        pytest.skip("the tensor-core pencil stage does not fit this grid")
    b.set_variant(pencil=0)
    sa = a.solve(a.initial_state(), 6)
    sb = b.solve(b.initial_state(), 6)
    for x, y in zip((*sa.u, sa.g), (*sb.u, sb.g), strict=True):
        assert rel(x, y.cpu().numpy()) < 1e-12


@pytest.mark.parametrize("N", [(17, 16, 16), (33, 32, 32), (65, 64, 64)])
def test_mixed_gradient_form_tracks_the_oracle(cuda, N):
    """Gradient form, mixed precision: complex64 periodic transforms of the
    products u_j d/dx_j u_i, the base-flow terms U_b d/dy u_i and
    u_0 dU_b/dx added in FP64 by the pencil stage; within 1e-7 of the FP64
    oracle after two startup and four steady SBDF3 steps."""
    kw = dict(nonlinear_form="gradient", time_integrator="SBDF3")
    o = PlaneCouetteOracle(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05, **kw)
    g = PlaneCouetteFluctuation(N=N, Re=400.0, dt=1e-3, perturbation_amplitude=0.05,
                                precision="mixed", device=cuda, **kw)
    st = o.initial_state()
    gs = g.solve(g._ensure_history(to_dev(st, cuda)), 6)
    st = o.solve(st, 6)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-7


@pytest.mark.parametrize("family", ["C", "L"])
def test_cnab2_rotational_keeps_laminar_state_and_matches_gradient_step(cuda, family):
    """The reference's CNAB2 property test
    (tests/couette/test_pcf_fluctuations_jax.py:104-136) on the GPU step:
    the laminar state stays zero, and one rotational step matches one
    gradient step (the forms differ by a pressure gradient)."""
    kw = dict(N=(13, 12, 12), family=family, dt=1.0e-4, padding_factor=(1.0, 1.5, 1.5),
              perturbation_amplitude=0.02, time_integrator="CNAB2", device=cuda)
    gradient = PlaneCouetteFluctuation(**kw, nonlinear_form="gradient")
    rotational = PlaneCouetteFluctuation(**kw, nonlinear_form="rotational")
    laminar = rotational.step(rotational.zero_state())
    for t in (*laminar.u, laminar.g):
        assert float(t.abs().max()) <= 2.0e-13
    gs = gradient.step(gradient.initial_state())
    rs = rotational.step(rotational.initial_state())
    for a, b in zip((*rs.u, rs.g), (*gs.u, gs.g), strict=True):
        assert torch.allclose(a, b, rtol=2.0e-7, atol=2.0e-10)


def test_mixed_gradient_form_has_no_tensor_core_velocity_variant(cuda, monkeypatch):
    """The tcgen05 velocity products form the rotational fields only: a
    gradient-form plan does not offer them, even when JFB200_TC asks."""
    monkeypatch.setenv("JFB200_TC", "1")
    g = PlaneCouetteFluctuation(N=(33, 32, 32), Re=400.0, dt=1e-3, precision="mixed",
                                nonlinear_form="gradient", time_integrator="SBDF3", device=cuda)
    v = g.variant()
    assert v["available"]["tc_velocity"] == 0 and v["current"]["tc_velocity"] == 0


@pytest.mark.parametrize("family", ["C", "L"])
@pytest.mark.parametrize("integrator", ["IMEXRK222", "CNAB2", "SBDF3"])
def test_smallest_grids_without_dealiasing_match_oracle(cuda, family, integrator):
    """The reference's small test grids (9, 4, 4) with padding (1, 1, 1):
    two-point Fourier half spectra and four-point transforms, gradient form,
    against the oracle after three steps."""
    kw = dict(family=family, nonlinear_form="gradient", time_integrator=integrator,
              padding_factor=(1.0, 1.0, 1.0))
    o = PlaneCouetteOracle(N=(9, 4, 4), Re=200.0, dt=1e-3, perturbation_amplitude=0.05, **kw)
    g = PlaneCouetteFluctuation(N=(9, 4, 4), Re=200.0, dt=1e-3, perturbation_amplitude=0.05,
                                device=cuda, **kw)
    st = o.initial_state()
    gs = g.solve(g._ensure_history(to_dev(st, cuda)), 3)
    st = o.solve(st, 3)
    for a, b in zip((*gs.u, gs.g), (*st.u, st.g), strict=True):
        assert rel(a, b) < 1e-12


def test_imaginary_mean_flow_input_steps_to_a_real_mean(cuda):
    """The reference's mean-mode test (tests/couette/test_pcf_fluctuations_jax.py:
    198-215): imaginary parts added to the (0, 0) modes of u1, u2 leave no
    imaginary part in the stepped mean flow."""
    g = PlaneCouetteFluctuation(N=(9, 4, 4), Re=200.0, dt=1e-3, padding_factor=(1.0, 1.0, 1.0),
                                device=cuda)
    s0 = g.initial_state()
    u1, u2 = s0.u[1].clone(), s0.u[2].clone()
    im = 1e-4j * torch.linspace(1.0, 2.0, u1.shape[0], dtype=torch.float64, device=cuda)
    u1[:, 0, 0] += im
    u2[:, 0, 0] += 2.0 * im
    s1 = g.step(KMMState(u=(s0.u[0], u1, u2), g=s0.g))
    assert float(s1.u[1][:, 0, 0].imag.abs().max()) < 1e-12
    assert float(s1.u[2][:, 0, 0].imag.abs().max()) < 1e-12


def test_zero_state_stays_zero(cuda):
    """tests/couette/test_pcf_fluctuations_jax.py:191-196: a step of the
    zero fluctuation (Legendre, default gradient form and integrator)."""
    g = PlaneCouetteFluctuation(N=(9, 8, 8), family="L", dt=1.0e-3, device=cuda)
    st = g.step(g.zero_state())
    for t in (*st.u, st.g):
        assert float(t.abs().max()) <= 1.0e-7
