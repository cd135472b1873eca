"""Standalone tensor-product transforms and the 2-D Helmholtz solver against
the oracle (GPU).  Transforms <= 1e-13 relative, the Helmholtz solution
<= 1e-12 relative (FP64)."""

import math

import numpy as np
import pytest
import torch

from jaxfun_b200.tps import Helmholtz2D, TensorProductSpace
from oracle import kmm as ok

pytestmark = pytest.mark.gpu

DOM3 = ((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi))


def rel(a, b):
    a = a.detach().cpu().numpy() if torch.is_tensor(a) else a
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def oracle_space(basis, N, family="C"):
    orth = ok.make_orthogonal(family, N[0], DOM3[0])
    x = orth if basis == "C" else ok.Composite1D(orth, "dirichlet" if basis == "D" else "biharmonic")
    return ok.TensorSpace(x, ok.Fourier1D(N[1], DOM3[1]), ok.Fourier1D(N[2], DOM3[2]))


@pytest.mark.parametrize("basis", ["C", "D", "B"])
@pytest.mark.parametrize("N", [(17, 16, 12), (33, 32, 32)])
def test_tps_transforms_match_oracle(cuda, basis, N):
    T = TensorProductSpace(basis, N, DOM3, padding_factor=(1.0, 1.5, 1.5), device=cuda)
    O = oracle_space(basis, N)
    rng = np.random.default_rng(5)
    c = rng.standard_normal(T.num_dofs) + 1j * rng.standard_normal(T.num_dofs)
    ct = torch.from_numpy(c).to(cuda)
    for padded in (False, True):
        counts = O.quad_counts((1.0, 1.5, 1.5)) if padded else O.quad_counts()
        assert rel(T.backward(ct, padded=padded), O.backward(c, counts)) < 1e-13, padded
    u = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ut = torch.from_numpy(u).to(cuda)
    assert rel(T.forward(ut), O.forward(u)) < 1e-13
    assert rel(T.scalar_product(ut), O.scalar_product(u)) < 1e-13
    # forward of a field sampled on the padded grid
    up = rng.standard_normal(O.quad_counts((1.0, 1.5, 1.5))).astype(complex)
    zo = up
    for ax in (2, 1, 0):
        zo = O.spaces[ax].forward(zo, axis=ax)
    assert rel(T.forward(torch.from_numpy(up).to(cuda), padded=True), zo) < 1e-13


def test_helmholtz2d_matches_dense_solve(cuda):
    """The 2-D Helmholtz case: N = 64 Chebyshev-Dirichlet x 64 Fourier,
    seeded forcing, against per-mode dense FP64 solves."""
    f_hat = ok.helmholtz2d_forcing((64, 64), seed=1)
    uh_ref, u_ref = ok.helmholtz2d_solve(f_hat)
    h = Helmholtz2D((64, 64), device=cuda)
    f_phys = h.TC.backward(torch.from_numpy(f_hat).to(cuda))
    assert rel(h.solve_coefficients(f_phys), uh_ref) < 1e-12
    u = h(torch.from_numpy(f_hat).to(cuda))
    assert rel(u, u_ref) < 1e-12
    assert float(torch.abs(u.imag).max()) < 1e-14 * float(torch.abs(u).max())


def test_helmholtz2d_manufactured_solution(cuda):
    """u = sum u_hat phi_j e^{iky}: f = -lap u + u is exact in the orthogonal
    basis, so the pipeline returns u_hat to round-off."""
    Nx, Ny = 32, 16
    rng = np.random.default_rng(9)
    orth = ok.make_orthogonal("C", Nx, (-1.0, 1.0))
    D = ok.Composite1D(orth, "dirichlet")
    uh = rng.standard_normal((Nx - 2, Ny)) + 1j * rng.standard_normal((Nx - 2, Ny))
    uh[:, Ny // 2] = 0
    k = np.fft.fftfreq(Ny, 1.0 / Ny)
    uo = D.to_orthogonal(uh, 0)
    f_hat = -orth.derivative_coeffs(uo, 2, 0) + (k[None, :] ** 2 + 1.0) * uo
    h = Helmholtz2D((Nx, Ny), device=cuda)
    f_phys = h.TC.backward(torch.from_numpy(f_hat).to(cuda))
    assert rel(h.solve_coefficients(f_phys), uh) < 1e-11


def test_helmholtz2d_graph_replay_matches_eager(cuda):
    f_hat = torch.from_numpy(ok.helmholtz2d_forcing((64, 64), seed=3)).to(cuda)
    h = Helmholtz2D((64, 64), device=cuda)
    eager = h(f_hat)
    g, f_in, u_out = h.graphed(f_hat)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(u_out, eager)
    f2 = torch.from_numpy(ok.helmholtz2d_forcing((64, 64), seed=4)).to(cuda)
    f_in.copy_(f2)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(u_out, h(f2))


@pytest.mark.parametrize("N", [(64, 64), (33, 48), (80, 32), (96, 96)])
def test_helmholtz2d_one_launch_matches_separate_launches(cuda, N):
    """jfb_helmholtz2d_solve (the whole pipeline in one CTA cluster) against the
    separate transforms and wavenumber solve, and against the oracle's
    per-mode dense solves."""
    h = Helmholtz2D(N, device=cuda)
    assert h.fused and h._Uinv is not None
    f_hat = ok.helmholtz2d_forcing(N, seed=5)
    f = torch.from_numpy(f_hat).to(cuda)
    one, sep = h(f), h.separate(f)
    assert rel(one, sep.cpu().numpy()) < 1e-12
    # the general form of the in-cluster solve (column-oriented substitution)
    h._Uinv = None
    assert rel(h(f), sep.cpu().numpy()) < 1e-12
    if N == (64, 64):
        _, u_ref = ok.helmholtz2d_solve(f_hat)
        assert rel(one, u_ref) < 1e-12


def test_helmholtz2d_too_large_for_one_cluster_uses_separate_launches(cuda):
    h = Helmholtz2D((144, 144), device=cuda)
    assert not h.fused
    f = torch.from_numpy(ok.helmholtz2d_forcing((144, 144), seed=6)).to(cuda)
    assert rel(h(f), h.separate(f).cpu().numpy()) == 0.0


def test_helmholtz2d_solve_rejects_mismatched_spaces(cuda):
    """The one-launch entry point checks its spaces and factors like the
    reference's solver construction (errors, no launch)."""
    from jaxfun_b200 import _lib

    h = Helmholtz2D((32, 16), device=cuda)
    f = torch.zeros((32, 16), dtype=torch.complex128, device=cuda)
    u = torch.empty((32, 16), dtype=torch.complex128, device=cuda)
    lo, uo = h._offs
    args = lambda tc, td: (tc._h, td._h, h._L.data_ptr(), lo, len(h.solver.L_offsets),  # noqa: E731
                           h._U.data_ptr(), uo, len(h.solver.U_offsets), None,
                           h._fourier_mass, f.data_ptr(), u.data_ptr(), None)
    with pytest.raises(_lib.JFBError) as e:  # Dirichlet space in the orthogonal slot
        _lib.call("jfb_helmholtz2d_solve", *args(h.TD, h.TD))
    assert e.value.status == _lib.JFB_ERR_ARG
    other = Helmholtz2D((33, 16), device=cuda)
    with pytest.raises(_lib.JFBError):  # sizes differ
        _lib.call("jfb_helmholtz2d_solve", *args(h.TC, other.TD))


@pytest.mark.parametrize("basis", ["C", "D", "B"])
@pytest.mark.parametrize("N", [(17, 16, 12), (33, 32, 32)])
def test_legendre_transforms_match_oracle(cuda, basis, N):
    """The Legendre family: Gauss-Legendre nodes and the dense Vandermonde
    contractions V @ c and (u w) @ V (orthogonal.py:121-145, 240-331)."""
    T = TensorProductSpace(basis, N, DOM3, padding_factor=(1.0, 1.5, 1.5), device=cuda,
                           family="L")
    O = oracle_space(basis, N, "L")
    rng = np.random.default_rng(7)
    c = rng.standard_normal(T.num_dofs) + 1j * rng.standard_normal(T.num_dofs)
    ct = torch.from_numpy(c).to(cuda)
    for padded in (False, True):
        counts = O.quad_counts((1.0, 1.5, 1.5)) if padded else O.quad_counts()
        assert rel(T.backward(ct, padded=padded), O.backward(c, counts)) < 1e-13, padded
    u = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ut = torch.from_numpy(u).to(cuda)
    assert rel(T.forward(ut), O.forward(u)) < 1e-13
    assert rel(T.scalar_product(ut), O.scalar_product(u)) < 1e-13
    # forward inverts backward on the space
    assert rel(T.forward(T.backward(ct)), c) < 1e-12
    if basis != "C":
        G0 = O.x.galerkin_matrix(0)
        assert np.abs(T.galerkin(0) - G0).max() <= 1e-13 * np.abs(G0).max()


@pytest.mark.parametrize("family", ["C", "L"])
@pytest.mark.parametrize("basis", ["C", "D", "B"])
def test_coefficient_space_maps_match_oracle(cuda, family, basis):
    """backward_primitive, to_orthogonal, differentiate_orthogonal_coeffs,
    project_from_orthogonal and scalar_product_from_orthogonal
    (tensorproductspace.py:553-754) against the oracle."""
    N = (25, 16, 12)
    T = TensorProductSpace(basis, N, DOM3, padding_factor=(1.0, 1.5, 1.5), device=cuda,
                           family=family)
    O = oracle_space(basis, N, family)
    rng = np.random.default_rng(11)
    c = rng.standard_normal(T.num_dofs) + 1j * rng.standard_normal(T.num_dofs)
    ct = torch.from_numpy(c).to(cuda)
    a = rng.standard_normal((N[0],) + N[1:]) + 1j * rng.standard_normal((N[0],) + N[1:])
    at = torch.from_numpy(a).to(cuda)
    for k in ((0, 0, 0), (1, 0, 0), (2, 1, 0), (0, 1, 2), (1, 3, 1)):
        for padded in (False, True):
            counts = O.quad_counts((1.0, 1.5, 1.5)) if padded else O.quad_counts()
            got = T.backward_primitive(ct, k, padded=padded)
            assert rel(got, O.backward_primitive(c, k, counts)) < 1e-12, (k, padded)
        assert rel(T.differentiate_orthogonal_coeffs(at, k),
                   O.differentiate_orthogonal_coeffs(a, k)) < 1e-12, k
        assert rel(T.derivative_orthogonal_coeffs(ct, k),
                   O.differentiate_orthogonal_coeffs(O.to_orthogonal(c), k)) < 1e-12, k
    assert rel(T.to_orthogonal(ct), O.to_orthogonal(c)) < 1e-14
    assert rel(T.project_from_orthogonal(at), O.project_from_orthogonal(a)) < 1e-13
    assert rel(T.scalar_product_from_orthogonal(at), O.scalar_product_from_orthogonal(a)) < 1e-13
    # project_from_orthogonal(to_orthogonal(c)) == c on the space
    assert rel(T.project_from_orthogonal(T.to_orthogonal(ct)), c) < 1e-13
