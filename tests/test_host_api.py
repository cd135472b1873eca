"""Host-side logic that needs no GPU: argument validation of the solver
objects, the workload generator and the benchmark's byte model."""

import math

import numpy as np
import pytest

import bench
from jaxfun_b200 import workloads
from jaxfun_b200.kmm import KMM, PlaneCouetteFluctuation


@pytest.mark.parametrize("kw", [
    {"dpdy": 0.1},
    {"padding_factor": (1.5, 1.5, 1.5)},
])
def test_unsupported_options_are_rejected_before_any_device_work(kw):
    with pytest.raises(NotImplementedError):
        KMM(N=(17, 16, 16), **kw)


@pytest.mark.parametrize("kw, exc", [
    ({"nonlinear_form": "skew"}, ValueError),
    ({"family": "J"}, ValueError),
    ({"coefficient_path": "fast"}, ValueError),
    ({"time_integrator": "RK4"}, ValueError),
])
def test_invalid_options_raise_value_error(kw, exc):
    with pytest.raises(exc):
        PlaneCouetteFluctuation(N=(17, 16, 16), **kw)


def test_workload_fields_are_divergence_free_and_wall_bounded():
    N = (33, 16, 16)
    dom = bench.domain()
    u0, u1, u2 = workloads.couette_perturbation_fields(N, dom)
    assert u0.shape == N and np.isfinite(u0).all()
    # no-slip: fields vanish towards the walls like (1 - x^2)
    x = np.cos(np.pi + (2 * np.arange(N[0]) + 1) * np.pi / (2 * N[0]))
    assert np.abs(u1[0]).max() < 10 * (1 - x[0] ** 2) * np.abs(u1).max()
    # spectral divergence of the analytic construction: d_y u1 + d_z u2 = 0 per x-plane
    # (u0 varies with x only through the envelope)
    Ly, Lz = dom[1][1] - dom[1][0], dom[2][1] - dom[2][0]
    ky = np.fft.fftfreq(N[1], 1.0 / N[1]) * 2 * np.pi / Ly
    kz = np.fft.fftfreq(N[2], 1.0 / N[2]) * 2 * np.pi / Lz
    f1, f2 = np.fft.fft2(u1), np.fft.fft2(u2)
    u0x = np.gradient(u0, x, axis=0, edge_order=2)
    div = np.fft.ifft2(1j * ky[None, :, None] * f1 + 1j * kz[None, None, :] * f2).real + u0x
    assert np.abs(div[N[0] // 2]).max() < 1e-2 * np.abs(u0x).max() + 1e-12
    s = workloads.scale_to_energy((u0,), 4.0, 1.0)[0]
    np.testing.assert_allclose(s, u0 * 0.5)


def test_stage_byte_model_matches_the_canonical_figure():
    sb = bench.stage_bytes((65, 64, 64), 96)
    # 43 E_s + 18 E_m complex at 16 B: 153.75 MB for 65x64x64
    assert abs(sb["step"] / 1e6 - 153.75) < 0.01
    fused = sum(sb[k] for k in ("pencil_stage", "y_backward", "z_cross", "y_forward"))
    assert fused < sb["step"]


def test_measured_peak_has_a_source():
    peak, kind = bench.measured_peak()
    assert peak > 1000 and kind in ("measured", "fallback")
    assert math.isfinite(peak)


def test_torch_library_ops_are_registered_with_fake_kernels():
    """The jaxfun_b200::* operators exist and their fake (meta) kernels give
    the output shapes without a GPU."""
    import torch
    from torch._subclasses.fake_tensor import FakeTensorMode

    from jaxfun_b200 import torch_ops  # noqa: F401

    ops = torch.ops.jaxfun_b200
    for name in ("dia_matvec", "wavenumber_solve", "tps_backward", "tps_forward", "kmm_gain"):
        assert hasattr(ops, name), name
    with FakeTensorMode():
        data = torch.empty((3, 9), dtype=torch.float64)
        x = torch.empty((4, 9, 2), dtype=torch.complex128)
        y = ops.dia_matvec(data, [-1, 0, 2], 11, 9, x, 1, False)
        assert tuple(y.shape) == (4, 11, 2) and y.dtype == torch.complex128
        z = ops.dia_matvec(data, [-1, 0, 2], 11, 9, torch.empty((11, 3)), 0, True)
        assert tuple(z.shape) == (9, 3)
        r = ops.wavenumber_solve(torch.empty((5, 1, 7)), [-2], torch.empty((5, 2, 7)), [0, 2],
                                 torch.empty((5, 7), dtype=torch.complex128))
        assert tuple(r.shape) == (5, 7)


def test_minimal_seed_ascent_rejects_bad_options():
    import pytest as _pytest

    from jaxfun_b200 import minimal_seed as ms

    for kw in (dict(steps=-1), dict(iterations=-2), dict(step_size=0.0),
               dict(min_step_size=float("inf")), dict(backtracking=1.0)):
        args = dict(steps=3, iterations=1, step_size=1.0, backtracking=0.5, min_step_size=1e-8)
        args.update(kw)
        with _pytest.raises(ValueError, match="minimal_seed_ascent"):
            ms._check_ascent_options(**args)
    assert ms._check_ascent_options(4, 2, 0.5, 0.5, 1e-8) == (4, 2)
    assert list(ms._TrialSteps(1.0, 0.5, 0.2)) == [1.0, 0.5, 0.25]


def test_checkpoint_payload_round_trip_keeps_every_history_level():
    """The production runner's payload layout (production/oracles.py:
    3872-3945, 327-420) for a flow state with SBDF3 / CNAB2 history and an
    MHD state: the restored state has the same arrays and scalars."""
    import torch

    from jaxfun_b200.checkpoint import (FLOW_KIND, MHD_KIND, checkpoint_payload,
                                        state_from_checkpoint_payload)
    from jaxfun_b200.kmm import KMMState
    from jaxfun_b200.mhd import MHDState

    g = torch.Generator().manual_seed(3)

    def arr(*shape):
        return torch.randn(*shape, 2, generator=g, dtype=torch.float64).contiguous()

    def lv():
        return (arr(5, 4, 4), arr(7, 4, 4), arr(7), arr(7))

    flow = KMMState(u=(arr(5, 4, 4), arr(7, 4, 4), arr(7, 4, 4)), g=arr(7, 4, 4),
                    nonlinear_old=lv(), nonlinear_older=lv(), solution_old=lv(),
                    solution_older=lv(), history_steps=2.0, have_old=1.0, previous_dt=0.01)
    back = state_from_checkpoint_payload(checkpoint_payload(flow), state_kind=FLOW_KIND)
    for name in ("u", "nonlinear_old", "nonlinear_older", "solution_old", "solution_older"):
        for a, b in zip(getattr(flow, name), getattr(back, name), strict=True):
            assert torch.equal(a, b)
    assert torch.equal(flow.g, back.g)
    assert (back.history_steps, back.have_old, back.previous_dt) == (2.0, 1.0, 0.01)

    cnab = KMMState(u=flow.u, g=flow.g, nonlinear_old=lv(), have_old=1.0, previous_dt=0.01)
    pl = checkpoint_payload(cnab)
    assert "solution_old" not in pl and pl["have_old"] == 1.0
    back = state_from_checkpoint_payload(pl, state_kind=FLOW_KIND)
    assert back.solution_old is None and back.nonlinear_older is None

    mhd = MHDState(flow=flow, A=(arr(7, 4, 4),) * 3, nonlinear_A_old=(arr(7, 4, 4),) * 3,
                   A_old=(arr(7, 4, 4),) * 3)
    pl = checkpoint_payload(mhd)
    assert "flow_u" in pl and "flow_history_steps" in pl and "A_older" not in pl
    back = state_from_checkpoint_payload(pl, state_kind=MHD_KIND)
    assert torch.equal(back.A[0], mhd.A[0]) and back.A_older is None
    assert torch.equal(back.flow.solution_older[1], flow.solution_older[1])
    with pytest.raises(ValueError):
        state_from_checkpoint_payload(pl, state_kind="axisymmetric_tc_hydro")
