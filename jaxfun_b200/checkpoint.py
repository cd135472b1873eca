"""Checkpoint payloads of the step's states (the production runner's layout).

The reference's runner turns a solver state into a flat payload of named
coefficient arrays before ``jaxfun.io.write_checkpoint`` stores it in HDF5,
and back again on resume (production/oracles.py:3872-3945 and 327-420).
These two functions produce and read the same keys for the states of this
package (``KMMState``: "pcf_fluctuation_saturation"; ``MHDState``:
"pcf_vector_potential_mhd_saturation"), so a resumed run carries the full
multistep history: the SBDF3 levels and ``history_steps``, CNAB2's
``nonlinear_old``, ``have_old`` and ``previous_dt``, and the A levels of the
MHD step.  Arrays stay torch tensors on their device; writing the payload to
a file is the caller's (the reference writes it with h5py).
"""

from __future__ import annotations

import torch

from .kmm import KMMState
from .mhd import MHDState

FLOW_KIND = "pcf_fluctuation_saturation"
MHD_KIND = "pcf_vector_potential_mhd_saturation"

_LEVELS = ("nonlinear_old", "nonlinear_older", "solution_old", "solution_older")


def _flow_payload(st: KMMState, prefix: str = "") -> dict:
    out = {f"{prefix}u": tuple(st.u), f"{prefix}g": st.g}
    if st.nonlinear_old is not None:
        out[f"{prefix}nonlinear_old"] = tuple(st.nonlinear_old)
        out[f"{prefix}have_old"] = float(st.have_old)
        out[f"{prefix}previous_dt"] = float(st.previous_dt)
    for name in _LEVELS[1:]:
        lv = getattr(st, name)
        if lv is not None:
            out[f"{prefix}{name}"] = tuple(lv)
    out[f"{prefix}history_steps"] = float(st.history_steps)
    return out


def _flow_state(payload: dict, prefix: str = "") -> KMMState:
    def level(name):
        v = payload.get(f"{prefix}{name}")
        return None if v is None else tuple(v)

    return KMMState(
        u=tuple(payload[f"{prefix}u"]),
        g=payload[f"{prefix}g"],
        nonlinear_old=level("nonlinear_old"),
        nonlinear_older=level("nonlinear_older"),
        solution_old=level("solution_old"),
        solution_older=level("solution_older"),
        history_steps=float(payload.get(f"{prefix}history_steps", 0.0)),
        have_old=float(payload.get(f"{prefix}have_old", 0.0)),
        previous_dt=float(payload.get(f"{prefix}previous_dt", 0.0)),
    )


def checkpoint_payload(state) -> dict:
    """Named arrays of a ``KMMState`` or ``MHDState``: the flow block as
    ``u, g, nonlinear_old, have_old, previous_dt, nonlinear_older,
    solution_old, solution_older, history_steps`` (present levels only), and
    for MHD the same with a ``flow_`` prefix plus ``A`` and its levels
    ``nonlinear_A_old, nonlinear_A_older, A_old, A_older``."""
    if isinstance(state, MHDState):
        out = _flow_payload(state.flow, "flow_")
        out["A"] = tuple(state.A)
        for name in ("nonlinear_A_old", "nonlinear_A_older", "A_old", "A_older"):
            lv = getattr(state, name)
            if lv is not None:
                out[name] = tuple(lv)
        return out
    if isinstance(state, KMMState):
        return _flow_payload(state)
    raise TypeError(f"no checkpoint layout for {type(state).__name__}")


def state_from_checkpoint_payload(payload: dict, *, state_kind: str):
    """The state a ``checkpoint_payload`` describes; ``state_kind`` as the
    reference's runner names it."""
    if state_kind == FLOW_KIND:
        return _flow_state(payload)
    if state_kind == MHD_KIND:
        def level(name):
            v = payload.get(name)
            return None if v is None else tuple(v)

        return MHDState(flow=_flow_state(payload, "flow_"), A=tuple(payload["A"]),
                        nonlinear_A_old=level("nonlinear_A_old"),
                        nonlinear_A_older=level("nonlinear_A_older"),
                        A_old=level("A_old"), A_older=level("A_older"))
    raise ValueError(f"unknown state_kind {state_kind!r}")


def payload_to_cpu(payload: dict) -> dict:
    """A copy of the payload with every tensor moved to host memory (what a
    file writer takes)."""
    def cpu(v):
        if torch.is_tensor(v):
            return v.detach().cpu()
        if isinstance(v, tuple):
            return tuple(cpu(x) for x in v)
        return v

    return {k: cpu(v) for k, v in payload.items()}
