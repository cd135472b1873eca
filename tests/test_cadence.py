"""Block splitting and callback order of ``run_with_cadence`` (host logic, no
GPU): the contract of src/jaxfun/io/__init__.py:97-183, with a counting
``advance`` in place of a plan's ``solve``."""

import pytest

from jaxfun_b200.cadence import Cadence, block_length, cadence_due, run_with_cadence


def counting_advance(log):
    def advance(state, n):
        log.append(n)
        return state + n

    return advance


def test_due_steps_and_cadence_due():
    c = Cadence(diagnostics_every=4, snapshot_every=None, checkpoint_every=0)
    assert c.due_steps() == (4,)
    assert Cadence(3, 5, 7).due_steps() == (3, 5, 7)
    assert cadence_due(8, 4) and not cadence_due(6, 4)
    assert not cadence_due(0, None) and not cadence_due(5, 0) and not cadence_due(5, -1)


def test_blocks_stop_at_every_boundary_and_the_final_step():
    log = []
    out = run_with_cadence(counting_advance(log), 0, steps=7, dt=0.5,
                           cadence=Cadence(diagnostics_every=2), block_size=3)
    assert out == 7
    assert log == [2, 2, 2, 1]
    # two cadences: boundaries at multiples of 3 and of 5
    assert [block_length(t, 20, Cadence(3, 5), 10) for t in (0, 3, 5, 6, 9, 10)] == [3, 2, 1, 3, 1, 2]
    # no cadence: blocks of block_size, the last one short
    log.clear()
    run_with_cadence(counting_advance(log), 0, steps=10, dt=1.0, cadence=Cadence(), block_size=4)
    assert log == [4, 4, 2]


def test_callbacks_order_time_and_offsets():
    events = []
    cad = Cadence(diagnostics_every=2, snapshot_every=3, checkpoint_every=6)
    out = run_with_cadence(
        counting_advance([]), 100, steps=6, dt=0.25, cadence=cad, block_size=10, t0=1.0, tstep0=4,
        diagnostics=lambda s: {"state": s},
        on_diagnostics=lambda t, k, d: events.append(("diag", t, k, d["state"])),
        on_snapshot=lambda t, k, s: events.append(("snap", t, k, s)),
        on_checkpoint=lambda t, k, s: events.append(("ckpt", t, k, s)),
    )
    assert out == 106
    # step counts 4 -> 10: boundaries 6 (2, 3 and 6 divide it), 8 (2), 9 (3), 10 (2)
    assert events == [
        ("diag", 1.5, 6, 102), ("snap", 1.5, 6, 102), ("ckpt", 1.5, 6, 102),
        ("diag", 2.0, 8, 104), ("snap", 2.25, 9, 105), ("diag", 2.5, 10, 106),
    ]


def test_diagnostics_none_and_missing_callbacks():
    got = []
    run_with_cadence(counting_advance([]), 0, steps=4, dt=1.0, cadence=Cadence(diagnostics_every=2),
                     on_diagnostics=lambda t, k, d: got.append((k, d)))
    assert got == [(2, None), (4, None)]
    # a due cadence without its callback changes only the block split
    log = []
    run_with_cadence(counting_advance(log), 0, steps=5, dt=1.0,
                     cadence=Cadence(checkpoint_every=2), block_size=5)
    assert log == [2, 2, 1]


def test_should_stop_ends_the_run_after_the_callbacks():
    events, log = [], []
    out = run_with_cadence(
        counting_advance(log), 0, steps=10, dt=1.0, cadence=Cadence(diagnostics_every=2),
        block_size=2, on_diagnostics=lambda t, k, d: events.append(k),
        should_stop=lambda t, k, s: k >= 4,
    )
    assert out == 4 and log == [2, 2] and events == [2, 4]


def test_zero_steps_and_argument_errors():
    log = []
    assert run_with_cadence(counting_advance(log), 5, steps=0, dt=1.0, cadence=Cadence(1)) == 5
    assert log == []
    with pytest.raises(ValueError, match="non-negative"):
        run_with_cadence(counting_advance(log), 0, steps=-1, dt=1.0, cadence=Cadence())
    with pytest.raises(ValueError, match="positive"):
        run_with_cadence(counting_advance(log), 0, steps=3, dt=1.0, cadence=Cadence(), block_size=0)
