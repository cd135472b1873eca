"""Resume from a checkpoint payload (the production runner's restart path).

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
