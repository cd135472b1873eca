"""Unit checks of the oracle's building blocks against independent NumPy
computations (CPU only)."""

from dataclasses import replace

import numpy as np
import pytest

from oracle import kmm as ok


@pytest.mark.parametrize("N", [9, 17, 33, 65])
def test_chebyshev_transforms_round_trip_and_nodes(N):
    c = ok.Chebyshev1D(N)
    rng = np.random.default_rng(N)
    coef = rng.standard_normal(N)
    u = c.backward(coef)
    V = np.polynomial.chebyshev.chebvander(c.nodes(), N - 1)
    np.testing.assert_allclose(u, V @ coef, atol=1e-13)
    np.testing.assert_allclose(c.forward(u), coef, atol=1e-13)
    # scalar products are exact Gauss-Chebyshev quadrature
    sp = c.scalar_product(u)
    np.testing.assert_allclose(sp, c.norm_squared() * coef, atol=1e-12)


@pytest.mark.parametrize("N", [9, 33])
def test_derivative_recurrences(N):
    rng = np.random.default_rng(1)
    coef = rng.standard_normal(N)
    ch = ok.Chebyshev1D(N).derivative_coeffs(coef, 2)
    ref = np.polynomial.chebyshev.chebder(coef, 2)
    np.testing.assert_allclose(ch[: ref.size], ref, atol=1e-10)
    lg = ok.Legendre1D(N).derivative_coeffs(coef, 1)
    ref = np.polynomial.legendre.legder(coef, 1)
    np.testing.assert_allclose(lg[: ref.size], ref, atol=1e-10)


@pytest.mark.parametrize("family", ["C", "L"])
def test_shen_bases_satisfy_boundary_conditions(family):
    orth = ok.make_orthogonal(family, 17)
    for bc, ders in (("dirichlet", (0,)), ("biharmonic", (0, 1))):
        comp = ok.Composite1D(orth, bc)
        for k in ders:
            rows = comp.boundary_rows(k)
            assert np.abs(rows).max() < 1e-12


def test_galerkin_matrices_match_quadrature():
    """(T_i, T_j^(k))_w by exact Gauss-Chebyshev quadrature of chebder."""
    N = 17
    c = ok.Chebyshev1D(N)
    x = c.nodes(N)
    w = np.full(N, np.pi / N)
    V = np.polynomial.chebyshev.chebvander(x, N - 1)
    for k in (0, 2, 4):
        Dk = np.zeros((N, N))
        for j in range(N):
            e = np.zeros(N)
            e[j] = 1
            d = np.polynomial.chebyshev.chebder(e, k) if k else e
            Dk[:, j] = V[:, : d.size] @ d
        quad = (V * w[:, None]).T @ Dk
        np.testing.assert_allclose(c.galerkin_matrix(k), quad, atol=1e-9 * np.abs(quad).max())


def test_banded_lu_matches_dense_solve():
    rng = np.random.default_rng(3)
    n, p, q = 21, 4, 8
    A = np.zeros((5, n, n))
    for b in range(5):
        for off in range(-p, q + 1, 2):
            A[b] += np.diag(rng.standard_normal(n - abs(off)), off)
        A[b] += np.eye(n) * 20
    lu = ok.BandedLU.factor(A)
    rhs = rng.standard_normal((5, n)) + 1j * rng.standard_normal((5, n))
    x = lu.solve(rhs)
    np.testing.assert_allclose(np.einsum("bij,bj->bi", A, x), rhs, atol=1e-12)


def test_wavenumber_solver_matches_kronecker_solve():
    """tests/la/test_tpmatrices_solvers.py:131-138 of the reference, on a
    Helmholtz system: per-mode solve vs the assembled Kronecker operator."""
    N = (9, 4, 6)
    D = ok.Composite1D(ok.Chebyshev1D(N[0]), "dirichlet")
    F1, F2 = ok.Fourier1D(N[1]), ok.Fourier1D(N[2])
    op = ok.mass_terms(D, F1, F2) - ok.laplace_terms(D, F1, F2).scale(0.1)
    solver = ok.WavenumberSolver(op)
    rng = np.random.default_rng(0)
    rhs = rng.standard_normal(solver.shape) + 1j * rng.standard_normal(solver.shape)
    x = solver.solve(rhs)
    np.testing.assert_allclose(op.matvec(x), rhs, atol=1e-10 * np.abs(rhs).max())


def test_sbdf3_third_order():
    """Third-order convergence of the SBDF3 combination on y' = -y + sin(t)
    split as implicit -y, explicit sin(t) (tests/integrators/test_sbdf3.py)."""
    def run(dt, T=2.0):
        n = int(round(T / dt))
        ex = lambda t: 0.5 * (np.sin(t) - np.cos(t)) + 1.5 * np.exp(-t)  # noqa: E731
        y = [ex(0.0), ex(dt), ex(2 * dt)]
        for k in range(2, n):
            t = k * dt
            nl = [np.sin(t), np.sin(t - dt), np.sin(t - 2 * dt)]
            rhs = (18 * y[-1] - 9 * y[-2] + 2 * y[-3]) / 11 + dt * (
                18 * nl[0] - 18 * nl[1] + 6 * nl[2]) / 11
            y.append(rhs / (1 + ok.SBDF3_IMPLICIT * dt))
        return abs(y[-1] - ex(n * dt))
    e1, e2 = run(0.02), run(0.01)
    order = np.log2(e1 / e2)
    assert 2.7 < order < 3.3


def test_fourier_padding_round_trip():
    f = ok.Fourier1D(16)
    rng = np.random.default_rng(2)
    c = rng.standard_normal(16) + 1j * rng.standard_normal(16)
    c[8] = 0
    u = f.backward(c, 24, 0)
    np.testing.assert_allclose(f.forward(u, 0), c, atol=1e-14)


def test_mhd_initial_magnetic_energy_is_analytic():
    """A_x = a (1 - x^2) sin(ky y) sin(kz z) / kz gives B = curl A =
    (0, a (1 - x^2) sin(ky y) cos(kz z), -a (ky / kz) (1 - x^2) cos(ky y) sin(kz z)),
    so Emag = a^2 (16/15) (Ly Lz / 4) (1 + (ky/kz)^2) exactly (1 - x^2 lies in
    the Dirichlet space)."""
    a = 0.2
    o = ok.PlaneCouetteMHDOracle(N=(17, 16, 16), Re=400.0, dt=1e-3, magnetic_amplitude=a)
    d = o.diagnostics(o.initial_state())
    Ly, Lz = 4.0 * np.pi, 2.0 * np.pi
    ky, kz = 2.0 * np.pi / Ly, 2.0 * np.pi / Lz
    exact = a * a * (16.0 / 15.0) * (Ly * Lz / 4.0) * (1.0 + (ky / kz) ** 2)
    assert abs(d["Emag"] - exact) < 1e-13 * exact
    assert d["divB_L2"] < 1e-15


def test_mhd_without_field_is_the_hydro_step():
    """magnetic_amplitude = 0: A stays zero, the flow follows the hydro oracle."""
    kw = dict(N=(17, 16, 16), Re=400.0, dt=1e-3, perturbation_amplitude=0.05)
    m = ok.PlaneCouetteMHDOracle(magnetic_amplitude=0.0, **kw)
    h = ok.PlaneCouetteOracle(**kw)
    sm, sh = m.solve(m.initial_state(), 4), h.solve(h.initial_state(), 4)
    for x, y in zip((*sm.flow.u, sm.flow.g), (*sh.u, sh.g), strict=True):
        np.testing.assert_allclose(x, y, rtol=0, atol=1e-16)
    assert all(np.abs(A).max() == 0.0 for A in sm.A)


def test_mhd_field_stays_solenoidal_and_couples():
    """B = curl A keeps div B at round-off through startup and steady steps,
    and the Lorentz force changes the flow."""
    kw = dict(N=(17, 16, 16), Re=400.0, dt=1e-3, perturbation_amplitude=0.05)
    m = ok.PlaneCouetteMHDOracle(magnetic_amplitude=0.5, **kw)
    st = m.solve(m.initial_state(), 5)
    assert m.magnetic_divergence_l2(st) < 1e-14
    h = ok.PlaneCouetteOracle(**kw)
    sh = h.solve(h.initial_state(), 5)
    assert np.linalg.norm(st.flow.u[0] - sh.u[0]) > 1e-8 * np.linalg.norm(sh.u[0])


@pytest.mark.parametrize("family", ["C", "L"])
def test_cnab2_laminar_state_and_form_agreement(family):
    """The reference's CNAB2 property test on the oracle
    (tests/couette/test_pcf_fluctuations_jax.py:104-136): the laminar state
    stays zero under the rotational form, the two forms' nonlinear rows Ng
    agree, and one rotational step matches one gradient step."""
    kw = dict(N=(13, 12, 12), family=family, dt=1.0e-4, padding_factor=(1.0, 1.5, 1.5),
              perturbation_amplitude=0.02, time_integrator="CNAB2")
    grad = ok.PlaneCouetteOracle(nonlinear_form="gradient", **kw)
    rot = ok.PlaneCouetteOracle(nonlinear_form="rotational", **kw)
    zero = rot.state_from_physical(tuple(np.zeros(rot.counts) for _ in range(3)))
    lam = rot.step(zero)
    for v in (*lam.u, lam.g):
        assert np.abs(v).max() <= 2.0e-13
    s0 = grad.initial_state()
    rg = grad.nonlinear_rhs(grad.convection(s0.u))
    rr = rot.nonlinear_rhs(rot.convection(s0.u))
    np.testing.assert_allclose(rr[1], rg[1], rtol=2.0e-11, atol=2.0e-12)
    a, b = grad.step(s0), rot.step(s0)
    for x, y in zip((*b.u, b.g), (*a.u, a.g), strict=True):
        np.testing.assert_allclose(x, y, rtol=2.0e-7, atol=2.0e-10)
    assert b.have_old == 1.0 and b.previous_dt == 1.0e-4


def test_cnab2_second_order_in_time():
    """Step-doubling order gate of the CNAB2 flow step (the reference's
    temporal-order gates, tests/couette/test_pcf_mri_cnab2_order_jax.py and
    tests/couette/test_pcf_sbdf3_jax.py:223-246, from a KMM-consistent
    initial state): the differences of runs at dt, dt/2, dt/4 to a common
    time shrink about fourfold."""
    T = 0.04

    def run(dt):
        s = ok.PlaneCouetteOracle(N=(13, 12, 12), Re=100.0, dt=dt, time_integrator="CNAB2",
                                  perturbation_amplitude=0.2, nonlinear_form="rotational")
        st = s.initial_state()
        means = (np.real(st.u[1][:, 0, 0]), np.real(st.u[2][:, 0, 0]))
        st = replace(st, u=s.reconstruct(st.u[0], st.g, *means))
        st = s.solve(st, int(round(T / dt)))
        return np.concatenate([st.u[0].ravel(), st.g.ravel(), st.u[1].ravel()])

    a, b, c = run(0.005), run(0.0025), run(0.00125)
    ratio = np.linalg.norm(a - b) / np.linalg.norm(b - c)
    assert 3.0 < ratio < 5.0
