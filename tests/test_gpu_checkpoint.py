"""Resume from a checkpoint payload, and the runner's cadence loop
(the production runner's restart and output path).

The reference checks that a run resumed from a checkpoint of its state,
history levels included, continues exactly as the uninterrupted run
(tests/couette/test_pcf_sbdf3_jax.py:170-187 for SBDF3, and
tests/production/test_pcf_cnab2_restart.py for CNAB2).  Here the payload
goes through host memory into a fresh plan.  The fresh plan forms the
nonlinear term of the loaded state anew (the uninterrupted plan kept the one
its last step produced), so the two continuations agree to round-off:
1e-13 relative L2 per field.
"""

import numpy as np
import pytest
import torch

from jaxfun_b200.cadence import Cadence
from jaxfun_b200.checkpoint import (FLOW_KIND, MHD_KIND, checkpoint_payload, payload_to_cpu,
                                    state_from_checkpoint_payload)
from jaxfun_b200.kmm import PlaneCouetteFluctuation
from jaxfun_b200.mhd import PlaneCouetteMHD

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = a.detach().cpu().numpy(), b.detach().cpu().numpy()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def to_device(payload, dev):
    def mv(v):
        if torch.is_tensor(v):
            return v.to(dev)
        if isinstance(v, tuple):
            return tuple(mv(x) for x in v)
        return v

    return {k: mv(v) for k, v in payload.items()}


@pytest.mark.parametrize("integrator, form", [("SBDF3", "rotational"), ("CNAB2", "gradient"),
                                              ("SBDF3", "gradient")])
def test_flow_restart_continues_the_run(cuda, integrator, form):
    kw = dict(N=(33, 32, 32), Re=400.0, dt=1e-3, perturbation_amplitude=0.05,
              time_integrator=integrator, nonlinear_form=form, device=cuda)
    parent = PlaneCouetteFluctuation(**kw)
    ck = parent.solve(parent.initial_state(), 4)
    payload = payload_to_cpu(checkpoint_payload(ck))
    restored = state_from_checkpoint_payload(to_device(payload, cuda), state_kind=FLOW_KIND)
    if integrator == "SBDF3":
        assert restored.history_steps == 2.0
    else:
        assert restored.have_old == 1.0 and restored.previous_dt == 1e-3
    expected = parent.solve(ck, 3)
    resumed = PlaneCouetteFluctuation(**kw).solve(restored, 3)
    for a, b in zip((*resumed.u, resumed.g), (*expected.u, expected.g), strict=True):
        assert rel(a, b) < 1e-13


def test_mhd_restart_continues_the_run(cuda):
    kw = dict(N=(33, 32, 32), Re=400.0, dt=1e-3, magnetic_amplitude=0.2, device=cuda)
    parent = PlaneCouetteMHD(**kw)
    ck = parent.solve(parent.initial_state(), 4)
    payload = payload_to_cpu(checkpoint_payload(ck))
    restored = state_from_checkpoint_payload(to_device(payload, cuda), state_kind=MHD_KIND)
    assert restored.flow.history_steps == 2.0
    expected = parent.solve(ck, 3)
    resumed = PlaneCouetteMHD(**kw).solve(restored, 3)
    a_ref = max(float(t.norm()) for t in expected.A)
    for a, b in zip((*resumed.flow.u, resumed.flow.g), (*expected.flow.u, expected.flow.g),
                    strict=True):
        assert rel(a, b) < 1e-13
    for a, b in zip(resumed.A, expected.A, strict=True):
        assert float((a - b).norm()) <= 1e-13 * a_ref


def test_solve_with_cadence_matches_direct_solve(cuda):
    """tests/couette/test_pcf_fluctuations_jax.py:258-281: one diagnostics
    event at step 2 and the same state as an uninterrupted solve."""
    kw = dict(N=(9, 4, 4), Re=200.0, dt=1e-3, padding_factor=(1.0, 1.0, 1.0), device=cuda)
    solver = PlaneCouetteFluctuation(**kw)
    state0 = solver.initial_state()
    events = []
    out = solver.solve_with_cadence(
        state0, 3, Cadence(diagnostics_every=2), block_size=2,
        on_diagnostics=lambda t, tstep, diag: events.append((t, tstep, diag["Epert"])))
    direct = PlaneCouetteFluctuation(**kw).solve(state0, 3)
    assert len(events) == 1 and events[0][1] == 2 and abs(events[0][0] - 2e-3) < 1e-15
    for a, b in zip((*out.u, out.g), (*direct.u, direct.g), strict=True):
        assert rel(a, b) < 1e-13


def test_cadence_checkpoints_resume_the_run(cuda):
    """The runner's loop: diagnostics and checkpoints at their cadences; the
    run resumed from the step-3 checkpoint in a fresh plan reaches the same
    state as the uninterrupted run."""
    kw = dict(N=(33, 32, 32), Re=400.0, dt=1e-3, perturbation_amplitude=0.05,
              time_integrator="SBDF3", nonlinear_form="gradient", device=cuda)
    solver = PlaneCouetteFluctuation(**kw)
    state0 = solver.initial_state()
    diags, ckpts = [], {}
    out = solver.solve_with_cadence(
        state0, 7, Cadence(diagnostics_every=2, checkpoint_every=3), block_size=5,
        on_diagnostics=lambda t, k, d: diags.append((k, d)),
        on_checkpoint=lambda t, k, s: ckpts.update({k: payload_to_cpu(checkpoint_payload(s))}))
    assert [k for k, _ in diags] == [2, 4, 6] and sorted(ckpts) == [3, 6]
    direct = PlaneCouetteFluctuation(**kw)
    at2 = direct.solve(state0, 2)
    ref2 = direct.diagnostics(at2)
    for name, v in diags[0][1].items():
        assert abs(v - ref2[name]) <= 1e-12 * max(1.0, abs(ref2[name])), name
    end = direct.solve(at2, 5)
    restored = state_from_checkpoint_payload(to_device(ckpts[3], cuda), state_kind=FLOW_KIND)
    resumed = PlaneCouetteFluctuation(**kw).solve_with_cadence(
        restored, 4, Cadence(diagnostics_every=2), block_size=4, tstep0=3, t0=3e-3)
    for a, b, c in zip((*out.u, out.g), (*end.u, end.g), (*resumed.u, resumed.g), strict=True):
        assert rel(a, b) < 1e-13 and rel(c, b) < 1e-13


def test_mhd_solve_with_cadence(cuda):
    kw = dict(N=(33, 32, 32), Re=400.0, dt=1e-3, magnetic_amplitude=0.2, device=cuda)
    solver = PlaneCouetteMHD(**kw)
    state0 = solver.initial_state()
    events = []
    out = solver.solve_with_cadence(state0, 4, Cadence(diagnostics_every=2), block_size=4,
                                    on_diagnostics=lambda t, k, d: events.append((k, d)))
    direct = PlaneCouetteMHD(**kw).solve(state0, 4)
    assert [k for k, _ in events] == [2, 4]
    assert set(events[0][1]) == set(solver.diagnostics(out))
    for a, b in zip((*out.flow.u, out.flow.g, *out.A),
                    (*direct.flow.u, direct.flow.g, *direct.A), strict=True):
        assert float((a - b).norm()) <= 1e-13 * max(float(b.norm()), 1e-30)
