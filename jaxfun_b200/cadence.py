"""Host-side cadence of a production run: blocks of device steps between
diagnostics, snapshot and checkpoint boundaries.

Same contract as the reference's ``jaxfun.io.Cadence`` /
``run_with_cadence`` (src/jaxfun/io/__init__.py:97-183), which
``KMM.solve_with_cadence`` (examples/channelflow_kmm.py:1264-1289) wraps and
the production runner calls (production/oracles.py:3293-3313):

* a block never crosses a step count that a positive cadence divides, nor
  the final step, and is at most ``block_size`` steps long;
* after each block the state is complete on the host's side (``solve`` of
  the B200 plans reads the device status word, which synchronises its
  stream), then, for the step count ``tstep`` reached and the time
  ``t = t0 + (tstep - tstep0) dt``, in this order: ``on_diagnostics(t,
  tstep, diagnostics(state))``, ``on_snapshot(t, tstep, state)``,
  ``on_checkpoint(t, tstep, state)``, each when its cadence divides
  ``tstep`` and the callback is given;
* ``should_stop(t, tstep, state)`` runs last and a true result ends the run
  before the next block.

The diagnostics are the plan's device reduction (``jfb_kmm_diagnostics``:
one launch, eight scalars read back), not a host computation on the state.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any, Callable


@dataclass(frozen=True)
class Cadence:
    """Step counts between diagnostics, snapshots and checkpoints (None or a
    non-positive value: never)."""

    diagnostics_every: int | None = None
    snapshot_every: int | None = None
    checkpoint_every: int | None = None

    def due_steps(self) -> tuple[int, ...]:
        """The positive cadences, in the order diagnostics, snapshot,
        checkpoint."""
        every = (self.diagnostics_every, self.snapshot_every, self.checkpoint_every)
        return tuple(int(e) for e in every if e is not None and e > 0)


def cadence_due(tstep: int, every: int | None) -> bool:
    """True when ``every`` is positive and divides ``tstep``."""
    return every is not None and every > 0 and tstep % every == 0


def block_length(tstep: int, final_tstep: int, cadence: Cadence, block_size: int) -> int:
    """Steps of the next block from ``tstep``: at most ``block_size``, and
    ending at the final step or the next step count a cadence divides,
    whichever comes first (at least one step while ``tstep < final_tstep``)."""
    n = min(int(block_size), final_tstep - tstep)
    for every in cadence.due_steps():
        n = min(n, every - tstep % every)  # in [1, every]
    return n


def run_with_cadence(
    advance: Callable[[Any, int], Any],
    state: Any,
    *,
    steps: int,
    dt: float,
    cadence: Cadence,
    block_size: int = 1,
    t0: float = 0.0,
    tstep0: int = 0,
    diagnostics: Callable[[Any], Any] | None = None,
    on_diagnostics: Callable | None = None,
    on_snapshot: Callable | None = None,
    on_checkpoint: Callable | None = None,
    should_stop: Callable | None = None,
) -> Any:
    """Advance ``state`` by ``steps`` steps of ``advance(state, n)`` in blocks,
    running the callbacks at the cadence boundaries; returns the last state.
    Raises ``ValueError`` for negative ``steps`` or ``block_size < 1``."""
    if steps < 0:
        raise ValueError("steps must be non-negative")
    if block_size < 1:
        raise ValueError("block_size must be positive")
    tstep, final_tstep = int(tstep0), int(tstep0) + int(steps)
    while tstep < final_tstep:
        n = block_length(tstep, final_tstep, cadence, block_size)
        state = advance(state, n)
        tstep += n
        t = float(t0) + (tstep - int(tstep0)) * float(dt)
        if on_diagnostics and cadence_due(tstep, cadence.diagnostics_every):
            on_diagnostics(t, tstep, None if diagnostics is None else diagnostics(state))
        if on_snapshot and cadence_due(tstep, cadence.snapshot_every):
            on_snapshot(t, tstep, state)
        if on_checkpoint and cadence_due(tstep, cadence.checkpoint_every):
            on_checkpoint(t, tstep, state)
        if should_stop is not None and bool(should_stop(t, tstep, state)):
            break
    return state
