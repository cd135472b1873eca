"""PyTorch custom operators (``torch.library``) over the C ABI.

The same sm_100a kernels that ``jaxfun_b200.la``, ``jaxfun_b200.tps`` and
``jaxfun_b200.kmm`` call through ctypes, registered as ``jaxfun_b200::*``
operators with fake (meta) implementations, so that they compose with
``torch.compile`` graph capture and ``torch.func`` tracing as opaque calls,
and with autograd formulas where the adjoint is available on the GPU:

* ``dia_matvec(data, offsets, n_rows, n_cols, x, axis, transpose)`` --
  ``DiaMatrix.matvec`` / ``rmatvec`` (src/jaxfun/la/diamatrix.py:227-348);
  its gradient is the transposed product (the matrix is real).
* ``wavenumber_solve(L, L_offsets, U, U_offsets, rhs)`` --
  ``TPMatricesWavenumberSolver.solve`` (src/jaxfun/la/tpmatrix.py:1550-1621)
  on a (n_F, n_P) right-hand side.
* ``tps_backward(handle, c, padded)`` / ``tps_forward(handle, u, padded,
  kind)`` -- ``TensorProductSpace.backward`` / ``forward`` /
  ``scalar_product`` (src/jaxfun/galerkin/tensorproductspace.py:253-293,
  529-551) of a space registered with ``register_space``.
* ``kmm_gain(handle, steps, checkpoint, u0, u1, u2, g)`` -- the perturbation
  gain E(T)/E(0) of ``pcf_minimal_seed_jax.py:111-122`` through ``steps``
  FP64 SBDF3 steps of a solver registered with ``register_solver``; its
  backward is the hand-written discrete adjoint (``jfb_kmm_gain_gradient``,
  PyTorch's complex convention: the conjugate of jax.grad's gradient).

Operators receive solvers and spaces as integer handles because
``torch.library`` schemas carry tensors and scalars only.
"""

from __future__ import annotations

import itertools

import torch

from . import _lib
from .la import DiaMatrix

_SOLVERS: dict[int, object] = {}
_SPACES: dict[int, object] = {}
_next = itertools.count(1)


def register_solver(solver) -> int:
    """Integer handle of a ``KMM`` / ``PlaneCouetteFluctuation`` solver for
    ``kmm_gain`` (kept alive until ``unregister``)."""
    h = next(_next)
    _SOLVERS[h] = solver
    return h


def register_space(space) -> int:
    """Integer handle of a ``TensorProductSpace`` for ``tps_backward`` /
    ``tps_forward``."""
    h = next(_next)
    _SPACES[h] = space
    return h


def unregister(handle: int) -> None:
    _SOLVERS.pop(int(handle), None)
    _SPACES.pop(int(handle), None)


def _lookup(table, handle, what):
    obj = table.get(int(handle))
    if obj is None:
        raise ValueError(f"no {what} registered under handle {handle}")
    return obj


# ---------------------------------------------------------------------------
# DIA matvec
# ---------------------------------------------------------------------------
def _dia_out_shape(x: torch.Tensor, n_rows: int, n_cols: int, axis: int, transpose: bool):
    shape = list(x.shape)
    shape[axis % x.dim()] = n_cols if transpose else n_rows
    return shape


@torch.library.custom_op("jaxfun_b200::dia_matvec", mutates_args=())
def dia_matvec(data: torch.Tensor, offsets: list[int], n_rows: int, n_cols: int,
               x: torch.Tensor, axis: int, transpose: bool) -> torch.Tensor:
    A = DiaMatrix(data, offsets, (n_rows, n_cols))
    return A._apply(x, axis, transpose)


@dia_matvec.register_fake
def _(data, offsets, n_rows, n_cols, x, axis, transpose):
    dt = torch.complex128 if x.is_complex() else torch.float64
    return x.new_empty(_dia_out_shape(x, n_rows, n_cols, axis, transpose), dtype=dt)


def _dia_setup(ctx, inputs, output):
    data, offsets, n_rows, n_cols, x, axis, transpose = inputs
    ctx.save_for_backward(data)
    ctx.meta = (list(offsets), n_rows, n_cols, axis, transpose, x.is_complex())


def _dia_backward(ctx, grad):
    (data,) = ctx.saved_tensors
    offsets, n_rows, n_cols, axis, transpose, cplx = ctx.meta
    g = dia_matvec(data, offsets, n_rows, n_cols, grad.contiguous(), axis, not transpose)
    if not cplx:
        g = g.real if g.is_complex() else g
    return None, None, None, None, g, None, None


dia_matvec.register_autograd(_dia_backward, setup_context=_dia_setup)


# ---------------------------------------------------------------------------
# Per-wavenumber banded solve
# ---------------------------------------------------------------------------
@torch.library.custom_op("jaxfun_b200::wavenumber_solve", mutates_args=())
def wavenumber_solve(L: torch.Tensor, L_offsets: list[int], U: torch.Tensor,
                     U_offsets: list[int], rhs: torch.Tensor) -> torch.Tensor:
    from .la import _stream

    if rhs.dim() != 2 or U.dim() != 3 or U.shape[0] != rhs.shape[0] or U.shape[2] != rhs.shape[1]:
        raise ValueError("rhs must be (n_F, n_P) and U (n_F, n_U, n_P)")
    n_F, n_P = rhs.shape
    cplx = rhs.is_complex()
    x = rhs.to(torch.complex128 if cplx else torch.float64).contiguous().clone()
    L = L.contiguous()
    _lib.call("jfb_wavenumber_solve", L.data_ptr() if L.numel() else None,
              _lib.int64_array(L_offsets), len(L_offsets), U.contiguous().data_ptr(),
              _lib.int64_array(U_offsets),
              len(U_offsets), n_P, n_F, 1, 1, x.data_ptr(), x.data_ptr(), int(cplx),
              _stream(x))
    return x


@wavenumber_solve.register_fake
def _(L, L_offsets, U, U_offsets, rhs):
    return rhs.new_empty(rhs.shape, dtype=torch.complex128 if rhs.is_complex() else torch.float64)


# ---------------------------------------------------------------------------
# Tensor-product transforms
# ---------------------------------------------------------------------------
@torch.library.custom_op("jaxfun_b200::tps_backward", mutates_args=())
def tps_backward(handle: int, c: torch.Tensor, padded: bool) -> torch.Tensor:
    return _lookup(_SPACES, handle, "space").backward(c, padded=padded)


@tps_backward.register_fake
def _(handle, c, padded):
    T = _lookup(_SPACES, handle, "space")
    return c.new_empty(T.padded_counts if padded else T.counts, dtype=torch.complex128)


@torch.library.custom_op("jaxfun_b200::tps_forward", mutates_args=())
def tps_forward(handle: int, u: torch.Tensor, padded: bool, kind: int) -> torch.Tensor:
    T = _lookup(_SPACES, handle, "space")
    return T.scalar_product(u, padded=padded) if kind else T.forward(u, padded=padded)


@tps_forward.register_fake
def _(handle, u, padded, kind):
    T = _lookup(_SPACES, handle, "space")
    return u.new_empty(T.num_dofs, dtype=torch.complex128)


# ---------------------------------------------------------------------------
# Perturbation gain with the hand-written adjoint as its backward
# ---------------------------------------------------------------------------
@torch.library.custom_op("jaxfun_b200::kmm_gain_fwd", mutates_args=())
def _kmm_gain_fwd(handle: int, steps: int, checkpoint: int, u0: torch.Tensor,
                  u1: torch.Tensor, u2: torch.Tensor, g: torch.Tensor) -> list[torch.Tensor]:
    """(gain, and the gradient leaves in PyTorch's convention) in one call."""
    from . import minimal_seed as ms
    from .kmm import KMMState

    solver = _lookup(_SOLVERS, handle, "solver")
    st = KMMState(u=(u0.contiguous(), u1.contiguous(), u2.contiguous()), g=g.contiguous())
    gain, grad = ms.gain_and_gradient(solver, st, steps, checkpoint=checkpoint)
    out = [torch.tensor(gain, dtype=torch.float64, device=u0.device)]
    out += [torch.conj(t).resolve_conj() for t in (*grad.u, grad.g)]
    return out


@_kmm_gain_fwd.register_fake
def _(handle, steps, checkpoint, u0, u1, u2, g):
    return [u0.new_empty((), dtype=torch.float64)] + [t.new_empty(t.shape) for t in (u0, u1, u2, g)]


@torch.library.custom_op("jaxfun_b200::kmm_gain", mutates_args=())
def kmm_gain(handle: int, steps: int, checkpoint: int, u0: torch.Tensor, u1: torch.Tensor,
             u2: torch.Tensor, g: torch.Tensor) -> torch.Tensor:
    from . import minimal_seed as ms
    from .kmm import KMMState

    solver = _lookup(_SOLVERS, handle, "solver")
    st = KMMState(u=(u0.contiguous(), u1.contiguous(), u2.contiguous()), g=g.contiguous())
    gain, _ = ms.gain_and_gradient(solver, st, steps, checkpoint=checkpoint,
                                   with_gradient=False)
    return torch.tensor(gain, dtype=torch.float64, device=u0.device)


@kmm_gain.register_fake
def _(handle, steps, checkpoint, u0, u1, u2, g):
    return u0.new_empty((), dtype=torch.float64)


def _gain_setup(ctx, inputs, output):
    ctx.args = inputs[:3]
    ctx.save_for_backward(*inputs[3:])


def _gain_backward(ctx, grad_out):
    handle, steps, checkpoint = ctx.args
    leaves = ctx.saved_tensors
    res = _kmm_gain_fwd(handle, steps, checkpoint, *leaves)
    return (None, None, None, *(grad_out * t for t in res[1:]))


kmm_gain.register_autograd(_gain_backward, setup_context=_gain_setup)
