"""jaxfun.la drop-ins on the GPU vs NumPy dense algebra and the oracle."""

import numpy as np
import pytest
import torch

from jaxfun_b200 import _lib
from jaxfun_b200.la import DiaMatrix, TPMatrices, TPMatrix, tpmats_wavenumber_factor
from oracle import kmm as ok

pytestmark = pytest.mark.gpu


def dense_dia(n, m, offsets, rng):
    a = np.zeros((n, m))
    for k in offsets:
        d = np.diagonal(a, k).size
        idx = np.arange(d)
        a[idx + max(0, -k), idx + max(0, k)] = rng.standard_normal(d)
    return a


@pytest.mark.parametrize("shape, offsets, axis", [
    ((7, 9), (-2, 0, 1, 3), 0), ((9, 7), (-3, 0, 2), 1), ((8, 8), (-1, 0, 1, 4), 2)])
@pytest.mark.parametrize("cplx", [False, True])
def test_matvec_rmatvec(cuda, shape, offsets, axis, cplx):
    rng = np.random.default_rng(0)
    a = dense_dia(*shape, offsets, rng)
    A = DiaMatrix.from_dense(torch.from_numpy(a).to(cuda), offsets)
    xs = [4, 5, 3]
    xs[axis] = shape[1]
    x = rng.standard_normal(xs) + (1j * rng.standard_normal(xs) if cplx else 0)
    y = A.matvec(torch.from_numpy(x).to(cuda), axis).cpu().numpy()
    ref = np.moveaxis(np.tensordot(a, np.moveaxis(x, axis, 0), axes=(1, 0)), 0, axis)
    np.testing.assert_allclose(y, ref, atol=1e-13)
    xs[axis] = shape[0]
    x = rng.standard_normal(xs) + (1j * rng.standard_normal(xs) if cplx else 0)
    y = A.rmatvec(torch.from_numpy(x).to(cuda), axis).cpu().numpy()
    ref = np.moveaxis(np.tensordot(a.T, np.moveaxis(x, axis, 0), axes=(1, 0)), 0, axis)
    np.testing.assert_allclose(y, ref, atol=1e-13)


def test_dia_solve_matches_oracle_lu(cuda):
    rng = np.random.default_rng(1)
    n = 31
    a = dense_dia(n, n, (-4, -2, 0, 2, 4, 6), rng) + 10 * np.eye(n)
    A = DiaMatrix.from_dense(torch.from_numpy(a).to(cuda), (-4, -2, 0, 2, 4, 6))
    b = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
    x = A.solve(torch.from_numpy(b).to(cuda), 0).cpu().numpy()
    ref = ok.BandedLU.factor(a).solve(b)
    np.testing.assert_allclose(x, ref, rtol=0, atol=1e-13 * np.abs(ref).max())


@pytest.mark.parametrize("cplx", [False, True])
def test_wide_factor_solve_matches_dense(cuda, cplx):
    """More than 32 diagonals on each side of the diagonal: the warp-per-system
    solve with its second pass over the diagonals (real and complex, several
    right-hand sides)."""
    rng = np.random.default_rng(3)
    n = 90
    offsets = tuple(range(-40, 0, 1)) + tuple(range(0, 70, 2))
    a = dense_dia(n, n, offsets, rng) * 0.05 + 4 * np.eye(n)
    A = DiaMatrix.from_dense(torch.from_numpy(a).to(cuda), offsets)
    b = rng.standard_normal((n, 5))
    if cplx:
        b = b + 1j * rng.standard_normal((n, 5))
    x = A.solve(torch.from_numpy(b).to(cuda), 0).cpu().numpy()
    ref = np.linalg.solve(a, b)
    np.testing.assert_allclose(x, ref, rtol=0, atol=1e-12 * np.abs(ref).max())


def test_singular_pivot_is_reported(cuda):
    a = np.eye(6)
    a[3, 3] = 0.0
    A = DiaMatrix.from_dense(torch.from_numpy(a).to(cuda), (0,))
    with pytest.raises(_lib.JFBError) as e:
        A.lu_factor()
    assert e.value.status == _lib.JFB_ERR_SINGULAR


def _helmholtz_tpmatrices(N, dev):
    D = ok.Composite1D(ok.Chebyshev1D(N[0]), "dirichlet")
    F1, F2 = ok.Fourier1D(N[1], (0, 4 * np.pi)), ok.Fourier1D(N[2])
    op = ok.mass_terms(D, F1, F2) - ok.laplace_terms(D, F1, F2).scale(0.05)
    tps = []
    for c, X, fy, fz in op.terms:
        mats = [DiaMatrix.from_dense(torch.from_numpy(X).to(dev)),
                DiaMatrix(torch.from_numpy(fy[None, :]).to(dev), (0,), (N[1], N[1])),
                DiaMatrix(torch.from_numpy(fz[None, :]).to(dev), (0,), (N[2], N[2]))]
        tps.append(TPMatrix(mats, c))
    return op, TPMatrices(tps)


def test_wavenumber_solver_matches_oracle_and_many_rhs(cuda):
    N = (33, 8, 12)
    op, A = _helmholtz_tpmatrices(N, cuda)
    solver = tpmats_wavenumber_factor(A)
    ref = ok.WavenumberSolver(op)
    rng = np.random.default_rng(2)
    rhs = rng.standard_normal(ref.shape) + 1j * rng.standard_normal(ref.shape)
    x = solver.solve(torch.from_numpy(rhs).to(cuda)).cpu().numpy()
    xr = ref.solve(rhs)
    np.testing.assert_allclose(x, xr, rtol=0, atol=1e-12 * np.abs(xr).max())
    assert solver.L_offsets == ref.lu.L_offsets and solver.U_offsets == ref.lu.U_offsets
    many = np.stack([rhs, 2 * rhs, rhs.conj()])
    xm = solver.solve_many(torch.from_numpy(many).to(cuda)).cpu().numpy()
    np.testing.assert_allclose(xm[1], 2 * xr, atol=1e-12 * np.abs(xr).max())
    L, U = solver.runtime_args()
    x2 = solver.solve_with_runtime_args(torch.from_numpy(rhs).to(cuda), (L, U)).cpu().numpy()
    np.testing.assert_array_equal(x2, x)
    # TPMatrices @ x reproduces the right-hand side
    back = (A @ torch.from_numpy(xr).to(cuda)).cpu().numpy()
    np.testing.assert_allclose(back, rhs, atol=1e-10 * np.abs(rhs).max())
