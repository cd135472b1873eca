"""Minimal-seed helpers on the sm_100a step and its hand-written adjoint.

Mirrors ``examples/pcf_minimal_seed_jax.py``: fixed-energy normalisation,
perturbation gain, its gradient (the discrete adjoint of the FP64 step in
``libjfb200.so``, ``jfb_kmm_gain_gradient``), the tangent projection on the
initial-energy constraint and the projected-gradient ascent loop.  Gradients
use jax.grad's convention for complex leaves: the directional derivative along
``d`` is ``Re(sum(g * d))``.  ``GainFunction`` wraps the same adjoint as a
``torch.autograd.Function`` (PyTorch's convention, ``conj(g)``).
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, replace

import torch

from . import _lib
from .kmm import KMM, KMMState

LEAVES = ("u", "g")


@dataclass(frozen=True)
class MinimalSeedIteration:
    """Record of one outer iteration of ``minimal_seed_ascent``.

    ``gain`` and ``energy`` belong to the iterate the gradient was taken at;
    ``step_size`` is the trial step that was taken (0.0 when none was), and
    ``accepted`` says whether the iterate moved."""

    iteration: int
    gain: float
    step_size: float
    gradient_norm: float
    energy: float
    accepted: bool


def _primary(state: KMMState) -> KMMState:
    """The differentiated leaves (u0, u1, u2, g) with a zero history."""
    return KMMState(u=tuple(state.u), g=state.g)


def tree_scale(state: KMMState, scale) -> KMMState:
    return KMMState(u=tuple(scale * u for u in state.u), g=scale * state.g)


def tree_add_scaled(state: KMMState, direction: KMMState, scale) -> KMMState:
    return KMMState(
        u=tuple(u + scale * du for u, du in zip(state.u, direction.u, strict=True)),
        g=state.g + scale * direction.g,
    )


def tree_conj(state: KMMState) -> KMMState:
    return KMMState(u=tuple(torch.conj(u).resolve_conj() for u in state.u),
                    g=torch.conj(state.g).resolve_conj())


def _leaves(state: KMMState):
    return (*state.u, state.g)


def tree_real_vdot(left: KMMState, right: KMMState) -> float:
    """``Re(sum(conj(left) * right))`` over the leaves."""
    return float(sum(torch.vdot(a.reshape(-1), b.reshape(-1)).real.item()
                     for a, b in zip(_leaves(left), _leaves(right), strict=True)))


def tree_l2_norm(state: KMMState) -> float:
    return math.sqrt(tree_real_vdot(state, state))


def jax_complex_directional_derivative(grad: KMMState, direction: KMMState) -> float:
    """``Re(sum(g * d))`` over the leaves (pcf_minimal_seed_jax.py:79-96)."""
    return float(sum(torch.sum(g * d).real.item()
                     for g, d in zip(_leaves(grad), _leaves(direction), strict=True)))


def _raise_if_not_positive(value: float, name: str) -> None:
    if not math.isfinite(value) or value <= 0.0:
        raise ValueError(f"{name} must be positive and finite")


def _empty_like(solver: KMM) -> KMMState:
    dev, cd = solver.device, torch.complex128
    return KMMState(
        u=(torch.empty(solver.shape_B, dtype=cd, device=dev),
           torch.empty(solver.shape_D, dtype=cd, device=dev),
           torch.empty(solver.shape_D, dtype=cd, device=dev)),
        g=torch.empty(solver.shape_D, dtype=cd, device=dev),
    )


def _c(solver: KMM, st: KMMState) -> _lib.KMMStateC:
    return solver._c_state(replace(st, history_steps=0.0))


def normalize_to_energy(solver: KMM, state: KMMState, target_energy: float) -> KMMState:
    """Rescale an initial condition to a target perturbation energy."""
    energy = solver.perturbation_energy(state)
    _raise_if_not_positive(energy, "state energy")
    _raise_if_not_positive(float(target_energy), "target energy")
    return tree_scale(_primary(state), math.sqrt(float(target_energy) / energy))


def perturbation_gain(solver: KMM, state: KMMState, steps: int) -> float:
    """Final perturbation energy divided by the initial one."""
    if int(steps) < 0:
        raise ValueError("steps must be non-negative")
    if int(steps) == 0:
        return 1.0
    return gain_and_gradient(solver, state, steps, with_gradient=False)[0]


def gain_and_gradient(solver: KMM, state: KMMState, steps: int, *, checkpoint: int = 20,
                      with_gradient: bool = True):
    """``jax.value_and_grad(perturbation_gain)`` through ``steps`` FP64 steps,
    recomputing ``checkpoint`` steps at a time in the reverse sweep."""
    if int(steps) < 1:
        raise ValueError("steps must be >= 1")
    st = _primary(state)
    gain = ctypes.c_double()
    grad = _empty_like(solver) if with_gradient else None
    _lib.call(
        "jfb_kmm_gain_gradient", solver._plan, ctypes.byref(_c(solver, st)), int(steps),
        int(checkpoint), ctypes.byref(gain),
        ctypes.byref(_c(solver, grad)) if grad is not None else None, solver._stream(),
    )
    solver._current = None
    return gain.value, grad


def energy_gradient(solver: KMM, state: KMMState) -> KMMState:
    """``jax.grad(solver.perturbation_energy)(state)``."""
    grad = _empty_like(solver)
    _lib.call("jfb_kmm_energy_gradient", solver._plan, ctypes.byref(_c(solver, _primary(state))),
              ctypes.byref(_c(solver, grad)), solver._stream())
    solver._current = None
    return grad


def project_to_energy_tangent(solver: KMM, state: KMMState, direction: KMMState) -> KMMState:
    """Project a direction onto the tangent space of constant initial energy
    (pcf_minimal_seed_jax.py:125-137)."""
    energy_grad = energy_gradient(solver, state)
    energy_normal = tree_conj(energy_grad)
    numerator = jax_complex_directional_derivative(energy_grad, direction)
    denominator = tree_real_vdot(energy_normal, energy_normal)
    _raise_if_not_positive(denominator, "energy-gradient norm")
    return tree_add_scaled(direction, energy_normal, -numerator / denominator)


def gain_and_projected_gradient(solver: KMM, state: KMMState, steps: int, *,
                                checkpoint: int = 20):
    """Perturbation gain and its gradient projected to fixed energy
    (pcf_minimal_seed_jax.py:140-150)."""
    gain, grad = gain_and_gradient(solver, state, steps, checkpoint=checkpoint)
    return gain, project_to_energy_tangent(solver, state, grad)


def _check_ascent_options(steps, iterations, step_size, backtracking, min_step_size):
    """Argument validation of ``minimal_seed_ascent``; returns the integer
    horizon and iteration count."""
    steps, iterations = int(steps), int(iterations)
    problems = []
    if steps < 0:
        problems.append(f"the horizon (steps={steps}) cannot be negative")
    if iterations < 0:
        problems.append(f"the iteration count ({iterations}) cannot be negative")
    for name, value in (("step_size", step_size), ("min_step_size", min_step_size)):
        if not (math.isfinite(float(value)) and float(value) > 0.0):
            problems.append(f"{name} has to be a finite number > 0 (got {value!r})")
    if not (0.0 < float(backtracking) < 1.0):
        problems.append(f"backtracking has to lie strictly inside (0, 1) (got {backtracking!r})")
    if problems:
        raise ValueError("minimal_seed_ascent: " + "; ".join(problems))
    return steps, iterations


class _TrialSteps:
    """Geometric sequence of trial step lengths ``first, first*r, ...`` down
    to (and including) the last one that is still >= ``floor``."""

    def __init__(self, first: float, ratio: float, floor: float):
        self.first, self.ratio, self.floor = float(first), float(ratio), float(floor)

    def __iter__(self):
        t = self.first
        while t >= self.floor:
            yield t
            t *= self.ratio


class _FixedEnergyLineSearch:
    """Backtracking search along a unit ascent direction on the sphere of
    fixed initial energy: every trial point is renormalised to the target
    energy and scored by its gain E(T)/E(0), evaluated by the forward step on
    the GPU; the first trial whose gain is finite and not below the current
    gain wins (the acceptance rule of pcf_minimal_seed_jax.py:207-223)."""

    def __init__(self, solver: KMM, steps: int, target_energy: float):
        self.solver, self.steps, self.target = solver, steps, float(target_energy)

    def point(self, origin: KMMState, direction: KMMState, length: float) -> KMMState:
        return normalize_to_energy(self.solver, tree_add_scaled(origin, direction, length),
                                   self.target)

    def run(self, origin: KMMState, direction: KMMState, gain_now: float, trials):
        for length in trials:
            cand = self.point(origin, direction, length)
            g = perturbation_gain(self.solver, cand, self.steps)
            if math.isfinite(g) and g >= gain_now:
                return length, cand
        return None, origin


def minimal_seed_ascent(solver: KMM, state: KMMState, *, target_energy: float, steps: int,
                        iterations: int = 10, step_size: float = 1.0, backtracking: float = 0.5,
                        min_step_size: float = 1.0e-8, tolerance: float = 1.0e-10,
                        checkpoint: int = 20):
    """Projected-gradient ascent of the gain at fixed initial energy
    (pcf_minimal_seed_jax.py:153-238).

    Each iteration takes the gain and its energy-projected gradient from the
    hand-written adjoint (``gain_and_projected_gradient``), stops when the
    gradient norm is at most ``tolerance``, and otherwise runs a backtracking
    line search along the normalised gradient that starts from the last
    accepted step length (``step_size`` at first), shrinks it by
    ``backtracking`` and gives up below ``min_step_size``; the loop ends at
    the first iteration whose search fails.  Returns the final iterate and
    one ``MinimalSeedIteration`` per iteration run."""
    steps, iterations = _check_ascent_options(steps, iterations, step_size, backtracking,
                                              min_step_size)
    search = _FixedEnergyLineSearch(solver, steps, target_energy)
    x = normalize_to_energy(solver, state, target_energy)
    length = float(step_size)
    records = []
    for it in range(iterations):
        gain, pgrad = gain_and_projected_gradient(solver, x, steps, checkpoint=checkpoint)
        gnorm = tree_l2_norm(pgrad)
        energy = solver.perturbation_energy(x)
        if not math.isfinite(gain) or not math.isfinite(gnorm):
            raise FloatingPointError(
                f"minimal_seed_ascent: iteration {it} gave gain={gain!r}, "
                f"projected-gradient norm={gnorm!r}")
        if gnorm <= tolerance:  # stationary on the energy sphere
            records.append(MinimalSeedIteration(it, gain, 0.0, gnorm, energy, False))
            break
        taken, x_next = search.run(x, tree_scale(pgrad, 1.0 / gnorm), gain,
                                   _TrialSteps(length, backtracking, min_step_size))
        records.append(MinimalSeedIteration(it, gain, taken or 0.0, gnorm, energy,
                                            taken is not None))
        if taken is None:
            break
        x, length = x_next, taken
    return x, tuple(records)


class GainFunction(torch.autograd.Function):
    """``gain = GainFunction.apply(solver, steps, checkpoint, u0, u1, u2, g)``:
    E(T)/E(0) with the adjoint as its backward (PyTorch complex convention:
    the gradient is the conjugate of jax.grad's)."""

    @staticmethod
    def forward(ctx, solver, steps, checkpoint, u0, u1, u2, g):
        st = KMMState(u=(u0.contiguous(), u1.contiguous(), u2.contiguous()), g=g.contiguous())
        gain, grad = gain_and_gradient(solver, st, steps, checkpoint=checkpoint)
        ctx.grads = tuple(torch.conj(t).resolve_conj() for t in (*grad.u, grad.g))
        return torch.tensor(gain, dtype=torch.float64, device=u0.device)

    @staticmethod
    def backward(ctx, grad_out):
        return (None, None, None, *(grad_out * t for t in ctx.grads))
