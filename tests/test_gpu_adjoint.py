"""The hand-written adjoint of the FP64 step against central finite
differences of the forward step (GPU).

Gain J = E(T)/E(0) through startup (IMEXRK3) and steady (SBDF3) steps; the
gradient's directional derivative Re sum(g d) must match
(J(x + eps d) - J(x - eps d)) / (2 eps) to 1e-6 relative along seeded
divergence-free directions and along directions that move each leaf
(u0, u1, u2, g) on its own.
"""

import math

import pytest
import torch

from jaxfun_b200 import minimal_seed as ms
from jaxfun_b200.kmm import KMMState, PlaneCouetteFluctuation
from jaxfun_b200.workloads import couette_perturbation_fields

pytestmark = pytest.mark.gpu


def direction(solver, seed):
    f = couette_perturbation_fields(solver.N, solver.domain, seeds=(seed, seed + 1))
    return ms._primary(solver.state_from_physical(f))


def scaled_to(d, ref):
    return ms.tree_scale(d, ms.tree_l2_norm(ref) / ms.tree_l2_norm(d))


def fd_check(solver, x0, d, steps, eps=1e-6, checkpoint=4):
    _, g = ms.gain_and_gradient(solver, x0, steps, checkpoint=checkpoint)
    adj = ms.jax_complex_directional_derivative(g, d)
    jp = ms.perturbation_gain(solver, ms.tree_add_scaled(x0, d, eps), steps)
    jm = ms.perturbation_gain(solver, ms.tree_add_scaled(x0, d, -eps), steps)
    fd = (jp - jm) / (2 * eps)
    return adj, fd


@pytest.mark.parametrize("N, steps", [((17, 16, 16), 8), ((33, 32, 32), 12)])
def test_gradient_matches_central_fd_divergence_free(cuda, N, steps):
    s = PlaneCouetteFluctuation(N=N, Re=400.0, dt=0.01, perturbation_amplitude=0.1, device=cuda,
                                time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = ms._primary(s.initial_state())
    for seed in (200, 203):
        d = scaled_to(direction(s, seed), x0)
        adj, fd = fd_check(s, x0, d, steps)
        assert abs(adj - fd) <= 1e-6 * max(abs(fd), 1e-12), (seed, adj, fd)


def test_gradient_matches_central_fd_per_leaf(cuda):
    """Each leaf on its own: u1, u2 and g enter the first nonlinear term and
    the means independently of the primary state."""
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = ms._primary(s.initial_state())
    full = direction(s, 210)
    z = lambda t: torch.zeros_like(t)  # noqa: E731
    dirs = [
        KMMState(u=(full.u[0], z(full.u[1]), z(full.u[2])), g=z(full.g)),
        KMMState(u=(z(full.u[0]), full.u[1], z(full.u[2])), g=z(full.g)),
        KMMState(u=(z(full.u[0]), z(full.u[1]), full.u[2]), g=z(full.g)),
        KMMState(u=(z(full.u[0]), z(full.u[1]), z(full.u[2])), g=full.g),
    ]
    # these directional derivatives are 1e-3 .. 1e-5 of the gain, so the FD
    # step is 1e-4 (at 1e-6 the FD quotient carries ~1e-9 absolute round-off)
    for k, d in enumerate(dirs):
        d = scaled_to(d, x0)
        adj, fd = fd_check(s, x0, d, 6, eps=1e-4)
        assert abs(adj - fd) <= 1e-6 * abs(fd), (k, adj, fd)


def test_checkpoint_stride_does_not_change_the_gradient(cuda):
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = ms._primary(s.initial_state())
    ga, a = ms.gain_and_gradient(s, x0, 9, checkpoint=1)
    gb, b = ms.gain_and_gradient(s, x0, 9, checkpoint=4)
    gc, c = ms.gain_and_gradient(s, x0, 9, checkpoint=9)
    assert ga == gb == gc
    for x, y, w in zip(ms._leaves(a), ms._leaves(b), ms._leaves(c), strict=True):
        assert torch.equal(x, y) and torch.equal(x, w)


def test_gain_matches_the_forward_solver(cuda):
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = s.initial_state()
    e0 = s.perturbation_energy(x0)
    eT = s.perturbation_energy(s.solve(x0, 7))
    gain, _ = ms.gain_and_gradient(s, x0, 7, with_gradient=False)
    assert abs(gain - eT / e0) <= 1e-13 * abs(gain)


def test_energy_tangent_projection_and_autograd(cuda):
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = ms._primary(s.initial_state())
    # the energy gradient is exact: E is quadratic, so FD is exact up to round-off
    d = scaled_to(direction(s, 220), x0)
    ge = ms.energy_gradient(s, x0)
    eps = 1e-4
    fd = (s.perturbation_energy(ms.tree_add_scaled(x0, d, eps))
          - s.perturbation_energy(ms.tree_add_scaled(x0, d, -eps))) / (2 * eps)
    assert abs(ms.jax_complex_directional_derivative(ge, d) - fd) <= 1e-9 * abs(fd)
    # projected directions keep the energy to first order
    pdir = ms.project_to_energy_tangent(s, x0, d)
    assert abs(ms.jax_complex_directional_derivative(ge, pdir)) <= 1e-10 * abs(fd)
    # torch.autograd: backward of the gain gives conj of the jax-convention gradient
    leaves = [t.clone().requires_grad_(True) for t in (*x0.u, x0.g)]
    gain = ms.GainFunction.apply(s, 5, 2, *leaves)
    gain.backward()
    _, g = ms.gain_and_gradient(s, x0, 5, checkpoint=2)
    for t, gj in zip(leaves, ms._leaves(g), strict=True):
        assert torch.allclose(t.grad, gj.conj(), rtol=0, atol=1e-13 * gj.abs().max().item())


def test_ascent_increases_gain_at_fixed_energy(cuda):
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = s.initial_state()
    final, hist = ms.minimal_seed_ascent(s, x0, target_energy=1e-4, steps=10, iterations=3,
                                         step_size=0.5)
    assert hist and all(math.isfinite(h.gain) for h in hist)
    assert abs(s.perturbation_energy(final) - 1e-4) <= 1e-12
    accepted = [h for h in hist if h.accepted]
    assert accepted
    assert ms.perturbation_gain(s, final, 10) >= hist[0].gain
