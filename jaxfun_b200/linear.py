"""Plane-Couette linear stability and transient growth on the KMM step's
Legendre-Galerkin operators, batched over wavenumbers on the GPU.

Mirrors the reference's dense linear tools for the hydrodynamic operator:
``jaxfun.la`` (src/jaxfun/la/eig.py: ``parse_times``, ``finite_eigenvalues``,
``finite_eigensystem``, ``generalized_eig``, ``physical_eigensystem``,
``transient_growth_from_eigs``) and ``PlaneCouetteLinear``
(examples/pcf_linear_jax.py: ``couette``, ``assemble``, ``energy_matrix``,
``eigs``, ``growth_rate``, ``nonmodal_growth``).

Discretisation.  The reference writes primitive variables (u_x, u_y, u_z, p)
as Chebyshev-Lobatto collocation values, a 4 nx x 4 nx descriptor pencil per
mode with wall rows of zero mass, and solves it by QZ on the host.  Here the
unknowns are those of the KMM step: the wall-normal velocity u in the
Legendre biharmonic basis (nx - 4 functions, u = u' = 0 at the walls) and
the wall-normal vorticity g = dy u_z - dz u_y in the Legendre Dirichlet basis
(nx - 2 functions), i.e. the bases of the step with ``family="L"``.  For a
Fourier mode exp(i ky y + i kz z), k^2 = ky^2 + kz^2, base flow
U(x) = Uoffset + Uprime x along y and rotation omega about z, Galerkin
projection of

    d/dt lap u = nu lap^2 u - i ky U lap u - 2 i omega kz g
    d/dt g     = nu lap g   - i ky U g    + i kz (Uprime + 2 omega) u

gives ``M dq/dt = L q`` with an invertible M (no eigenvalues at infinity) of
order 2 nx - 6.  The kinetic energy of the mode is
q^H Q q, Q = diag(A0 + A1 / k^2, B0 / k^2) (u_y, u_z follow from continuity
and g).  The physical eigenvalues and growth agree with the reference's to
its printed digits (the tests compare both with its recorded outputs).

Device work (torch on the GPU): the per-mode operators of a batch of
wavenumbers are formed in one pass from nine fixed basis matrices; the
eigenvalues come from the shift-inverted ``L^-1 M`` (batched solve and
eigen-decomposition of the cuSOLVER-backed ``torch.linalg``), which resolves
the least damped modes to relative accuracy; the optimal growth of all requested
times is one batched matrix exponential ``exp(A t)`` and one batched
singular-value call, G(t) = || R exp(A t) R^-1 ||_2^2 with R the Cholesky
factor of Q, which needs no eigenvectors.  The eigenvector route of
``transient_growth_from_eigs`` (the reference's) serves ``n_modes``
truncations.

MHD (``mhd=True``, ``shearpy``): the induction equation with an imposed
field (0, by, bz), the magnetic multiplier of div b = 0 and the four
magnetic wall conditions (conducting, dirichlet, pseudo_vacuum, insulating)
are wall rows of a descriptor pencil; here that operator keeps the
reference's primitive-variable Chebyshev-Lobatto form (eight blocks of nx
values), assembled for a batch of modes on the device, with the same
shift-inverted eigen-solve (a singular M maps to infinite eigenvalues, which
the finite cap removes) and the reference's modal route for the transient
growth in the kinetic, magnetic or total energy.
"""

from __future__ import annotations

import math

import numpy as np
import torch
from numpy.polynomial import legendre as npleg

MODAL_FINITE_CAP = 1.0e6
NONMODAL_FINITE_CAP = 1.0e8

_MAGNETIC_BCS = ("conducting", "dirichlet", "pseudo_vacuum", "insulating")


# ----------------------------------------------------------------------------
# eigen helpers (src/jaxfun/la/eig.py), on torch tensors
# ----------------------------------------------------------------------------

def parse_times(value) -> np.ndarray:
    """Times from a comma/semicolon separated string or a sequence
    (la/eig.py:22-35): at least one, none negative."""
    if isinstance(value, str):
        vals = [float(s) for s in value.replace(";", ",").split(",") if s.strip()]
    else:
        vals = [float(v) for v in (value.tolist() if torch.is_tensor(value) else list(value))]
    if not vals:
        raise ValueError("at least one time is required")
    out = np.asarray(vals, dtype=float)
    if (out < 0).any():
        raise ValueError("non-modal times must be non-negative")
    return out


def _tensor(a, device=None) -> torch.Tensor:
    if torch.is_tensor(a):
        t = a if device is None else a.to(device)
    else:
        t = torch.as_tensor(np.asarray(a), device=device or "cuda")
    return t.to(torch.complex128)


def _growth_sort(w: torch.Tensor) -> torch.Tensor:
    """Indices ordering ``w`` by descending real part, ties by descending
    imaginary part (la/eig.py:12-19)."""
    if w.numel() == 0:
        return torch.zeros(0, dtype=torch.long, device=w.device)
    by_imag = torch.argsort(-w.imag, stable=True)
    return by_imag[torch.argsort(-w.real[by_imag], stable=True)]


def _pencil_eig(L: torch.Tensor, M: torch.Tensor, vectors: bool = True):
    """Eigenvalues (and eigenvectors) of ``L q = s M q`` (batched over leading
    dimensions) by a shift-invert reduction: (L - sigma M)^-1 M v = mu v,
    s = sigma + 1/mu.  Directions that M maps to zero give mu = 0 and
    s = inf; eigenvalues near the shift come out with relative accuracy
    (the least damped modes of a stable operator, with sigma = 0, where the
    plain M^-1 L would lose digits to the large damped ones).  Shifts are
    tried until L - sigma M is regular."""
    n = L.shape[-1]
    scale = float(torch.linalg.matrix_norm(L, ord=1).max()) or 1.0
    for sigma in (0.0, 0.37 + 0.21j, -0.61 + 0.53j, 1.9 - 0.8j):
        s = complex(sigma) * scale / max(n, 1)
        X, info = torch.linalg.solve_ex(L - s * M, M)
        if int(info.max()) == 0 and bool(torch.isfinite(X).all()):
            if vectors:
                mu, V = torch.linalg.eig(X)
            else:
                mu, V = torch.linalg.eigvals(X), None
            inf = torch.tensor(complex(math.inf, 0.0), dtype=mu.dtype, device=mu.device)
            lam = torch.where(mu.abs() > 0, s + 1.0 / torch.where(mu.abs() > 0, mu, 1.0), inf)
            return lam, V
    raise ValueError("singular pencil: L - sigma M is singular for every trial shift")


def _keep_finite(w, V, finite_cap):
    keep = torch.isfinite(w.real) & torch.isfinite(w.imag) & (w.abs() < finite_cap)
    idx = torch.nonzero(keep).flatten()
    return w[idx], (None if V is None else V[:, idx])


def finite_eigenvalues(eigenvalues, *, finite_cap: float = MODAL_FINITE_CAP, sort: bool = True):
    """Finite eigenvalues below ``finite_cap``, growth-sorted (la/eig.py:38-54)."""
    w = _tensor(eigenvalues)
    w, _ = _keep_finite(w, None, finite_cap)
    return w[_growth_sort(w)] if sort else w


def generalized_eig(L, M, *, vectors: bool = False, finite_cap: float = MODAL_FINITE_CAP,
                    sort: bool = True, device=None):
    """Finite eigenvalues (and unit-norm eigenvectors) of ``L q = s M q``
    (la/eig.py:166-194)."""
    Lt = _tensor(L, device)
    w, V = _pencil_eig(Lt, _tensor(M, Lt.device))
    w, V = _keep_finite(w, V, finite_cap)
    if sort and w.numel():
        o = _growth_sort(w)
        w, V = w[o], V[:, o]
    return (w, V) if vectors else w


def finite_eigensystem(L, M, *, finite_cap: float = NONMODAL_FINITE_CAP, n_return=None, device=None):
    """Growth-sorted finite eigenpairs (la/eig.py:57-77)."""
    w, V = generalized_eig(L, M, vectors=True, finite_cap=finite_cap, sort=True, device=device)
    if n_return is not None:
        w, V = w[:n_return], V[:, :n_return]
    return w, V


def physical_eigensystem(L, M, metric, *, finite_cap: float = NONMODAL_FINITE_CAP, n_return=None,
                         metric_rtol=None, device=None):
    """Finite eigenpairs whose eigenvector carries energy under ``metric``:
    q^H Q q > rtol ||Q||_2 |q|^2, rtol = sqrt(eps) by default
    (la/eig.py:197-242)."""
    tol = math.sqrt(np.finfo(float).eps) if metric_rtol is None else float(metric_rtol)
    if not math.isfinite(tol) or tol < 0.0:
        raise ValueError("metric_rtol must be finite and nonnegative")
    w, V = finite_eigensystem(L, M, finite_cap=finite_cap, device=device)
    Q = _tensor(metric, V.device)
    if tuple(Q.shape) != (V.shape[0], V.shape[0]):
        raise ValueError(f"energy metric must have shape {(V.shape[0],) * 2}, got {tuple(Q.shape)}")
    if V.shape[1] == 0:
        return w, V
    scale = float(torch.linalg.matrix_norm(Q, ord=2))
    if not math.isfinite(scale) or scale <= 0.0:
        raise ValueError("energy metric must have a finite positive scale")
    energy = torch.einsum("im,im->m", V.conj(), Q @ V).real
    keep = torch.nonzero(energy > tol * scale * (V.abs() ** 2).sum(0)).flatten()
    w, V = w[keep], V[:, keep]
    if n_return is not None:
        w, V = w[:n_return], V[:, :n_return]
    return w, V


def _growth_rows(times, gains):
    return [{"t": float(t), "gain": float(g), "amplification": math.sqrt(float(g))}
            for t, g in zip(times, gains, strict=True)]


def transient_growth_from_eigs(evals, evecs, metric, times, *, metric_rtol: float = 1.0e-10):
    """Optimal growth G(t) of q(t) = V exp(Lambda t) a in the energy norm of
    ``metric`` (la/eig.py:80-124): with V^H Q V = U diag(d) U^H restricted
    to d > rtol max d, G(t) = || diag(sqrt d) U^H exp(Lambda t) U
    diag(1/sqrt d) ||_2^2.  All times in one batched singular-value call."""
    lam = _tensor(evals)
    V = _tensor(evecs, lam.device)
    Q = _tensor(metric, lam.device)
    times = parse_times(times)
    if lam.numel() == 0 or V.numel() == 0:
        raise ValueError("no finite eigenvectors available for non-modal growth")
    G = V.mH @ Q @ V
    d, U = torch.linalg.eigh(0.5 * (G + G.mH))
    big = float(d.abs().max())
    keep = torch.nonzero(d > max(metric_rtol * big, float(np.finfo(float).eps))).flatten()
    if keep.numel() == 0:
        raise ValueError("energy metric is singular on all retained modes")
    d, U = d[keep], U[:, keep]
    sq = torch.sqrt(d).to(U.dtype)
    F = sq[:, None] * U.mH                                                 # (r, m)
    tt = torch.as_tensor(times, dtype=torch.float64, device=lam.device)
    E = torch.exp(lam[None, :] * tt[:, None])                             # (T, m)
    P = (F[None] @ (E[:, :, None] * U[None])) / sq[None, None, :]         # (T, r, r)
    gains = (torch.linalg.svdvals(P)[:, 0] ** 2).cpu().numpy()
    return _growth_rows(times, gains)


def print_eigenvalues(evals, header: str = "leading eigenvalues") -> None:
    print(header)
    for v in (evals.tolist() if torch.is_tensor(evals) else list(evals)):
        v = complex(v)
        print(f"   s = {v.real:+.6e}  {v.imag:+.6e} i")


def print_transient_growth(rows, header: str = "non-modal transient growth") -> None:
    print(header)
    for r in rows:
        print(f"   t={r['t']:.6g}  G={r['gain']:.6e}  sqrt(G)={r['amplification']:.6e}")


# ----------------------------------------------------------------------------
# the KMM step's Legendre bases and their Galerkin matrices
# ----------------------------------------------------------------------------

def legendre_kmm_matrices(nx: int) -> dict[str, np.ndarray]:
    """Galerkin matrices of the Legendre biharmonic basis phi_k = L_k +
    a_k L_{k+2} + b_k L_{k+4} (a_k = -2(2k+5)/(2k+7), b_k = (2k+3)/(2k+7),
    k < nx - 4) and the Dirichlet basis psi_k = L_k - L_{k+2} (k < nx - 2),
    by Gauss-Legendre quadrature on nx + 2 nodes (exact: every integrand is a
    polynomial of degree <= 2 nx - 1):

    A0 = (phi_i, phi_j), A1 = (phi_i', phi_j'), A2 = (phi_i'', phi_j''),
    X0 = (phi_i, x phi_j), XD2 = (phi_i, x phi_j''), B0 = (psi_i, psi_j),
    B1 = (psi_i', psi_j'), XB = (psi_i, x psi_j), C = (psi_i, phi_j)."""
    nx = int(nx)
    if nx < 6:
        raise ValueError("nx must be at least 6 (two biharmonic functions)")
    nB, nD = nx - 4, nx - 2
    x, w = npleg.leggauss(nx + 2)
    V0 = npleg.legvander(x, nx - 1)
    Dc = np.zeros((nx, nx))
    for j in range(1, nx):
        e = np.zeros(j + 1)
        e[j] = 1.0
        d = npleg.legder(e)
        Dc[: d.size, j] = d
    V1 = V0 @ Dc
    V2 = V1 @ Dc
    k = np.arange(nB, dtype=float)
    SB = np.zeros((nB, nx))
    SB[np.arange(nB), np.arange(nB)] = 1.0
    SB[np.arange(nB), np.arange(nB) + 2] = -2.0 * (2 * k + 5) / (2 * k + 7)
    SB[np.arange(nB), np.arange(nB) + 4] = (2 * k + 3) / (2 * k + 7)
    SD = np.zeros((nD, nx))
    SD[np.arange(nD), np.arange(nD)] = 1.0
    SD[np.arange(nD), np.arange(nD) + 2] = -1.0
    P0, P1, P2 = V0 @ SB.T, V1 @ SB.T, V2 @ SB.T
    Q0, Q1 = V0 @ SD.T, V1 @ SD.T

    def ip(a, b, weight=w):
        return a.T @ (weight[:, None] * b)

    return {
        "A0": ip(P0, P0), "A1": ip(P1, P1), "A2": ip(P2, P2),
        "X0": ip(P0, P0, w * x), "XD2": ip(P0, P2, w * x),
        "B0": ip(Q0, Q0), "B1": ip(Q1, Q1), "XB": ip(Q0, Q0, w * x),
        "C": ip(Q0, P0),
    }


def cheb_lobatto(n: int):
    """Chebyshev-Lobatto points x_j = cos(pi j / (n-1)) (x_0 = +1), the
    collocation first-derivative matrix (diagonal from the negative row sums)
    and its square, and the Clenshaw-Curtis weights (Trefethen, Spectral
    Methods in MATLAB, cheb and clencurt)."""
    n = int(n)
    if n < 4:
        raise ValueError("nx must be at least 4")
    N = n - 1
    j = np.arange(n)
    theta = np.pi * j / N
    x = np.cos(theta)
    c = np.where((j == 0) | (j == N), 2.0, 1.0) * np.where(j % 2 == 0, 1.0, -1.0)
    D = np.outer(c, 1.0 / c) / (x[:, None] - x[None, :] + np.eye(n))
    D -= np.diag(D.sum(axis=1))
    s = np.ones(n)
    for k in range(1, N // 2 + 1):
        s -= (1.0 if 2 * k == N else 2.0) * np.cos(2 * k * theta) / (4.0 * k * k - 1.0)
    w = 2.0 * s / N
    w[0] = w[-1] = 1.0 / (N * N - 1.0) if N % 2 == 0 else 1.0 / (N * N)
    return x, D, D @ D, w


class PlaneCouetteLinear:
    """Plane-Couette linear operator on the KMM unknowns (u, g), batched
    over wavenumbers (examples/pcf_linear_jax.py:69-397, hydrodynamic part).

    Coordinates as the step: x wall-normal on [-1, 1], y streamwise, z
    spanwise; base flow U(x) = Uoffset + Uprime x along y, rotation
    ``omega`` about z.  ``ky``/``kz`` arguments accept scalars or arrays
    (broadcast together) wherever a batch makes sense.  Eigenvectors are
    coefficient vectors [u (nx - 4); g (nx - 2)] of the hydrodynamic
    operator, and collocation values of (u_x, u_y, u_z, p, b_x, b_y, b_z,
    phi) for the MHD operator (``mhd=True``)."""

    def __init__(self, nx=64, nu=1.0e-3, eta=1.0e-3, Uprime=1.0, Uoffset=0.0, omega=0.0,
                 by=0.0, bz=0.0, mhd=False, magnetic_bc="conducting", device="cuda"):
        if magnetic_bc not in _MAGNETIC_BCS:
            raise ValueError("magnetic_bc must be 'conducting', 'dirichlet', 'pseudo_vacuum' "
                             "or 'insulating'")
        self.nx, self.nu, self.eta = int(nx), float(nu), float(eta)
        self.Uprime, self.Uoffset, self.omega = float(Uprime), float(Uoffset), float(omega)
        self.by, self.bz, self.mhd, self.magnetic_bc = float(by), float(bz), bool(mhd), magnetic_bc
        self.device = torch.device(device)
        if self.mhd:
            x, D, D2, w = cheb_lobatto(self.nx)
            self._c = {k: torch.as_tensor(v, dtype=torch.complex128, device=self.device)
                       for k, v in (("x", x), ("D", D), ("D2", D2), ("w", w))}
            self.n = 8 * self.nx
            return
        self.nB, self.nD = self.nx - 4, self.nx - 2
        self.n = self.nB + self.nD
        mats = legendre_kmm_matrices(self.nx)
        self._m = {k: torch.as_tensor(v, dtype=torch.complex128, device=self.device)
                   for k, v in mats.items()}

    @classmethod
    def couette(cls, nx=64, Re=400.0, Rm=None, U_wall=1.0, mhd=False, **kw):
        """Couette flow between walls moving at -/+ U_wall (pcf_linear_jax.py:141-152)."""
        Rm = Re if Rm is None else Rm
        return cls(nx=nx, nu=float(U_wall) / float(Re), eta=float(U_wall) / float(Rm),
                   Uprime=float(U_wall), Uoffset=0.0, mhd=mhd, **kw)

    @classmethod
    def shearpy(cls, nx=64, Re=1000.0, Rm=1000.0, shear_rate=1.0, omega=2.0 / 3.0, by=0.0,
                bz=0.025, velocity_scale=1.0, **kw):
        """The rotating-shear MHD configuration (pcf_linear_jax.py:154-178)."""
        return cls(nx=nx, nu=float(velocity_scale) / float(Re), eta=float(velocity_scale) / float(Rm),
                   Uprime=-float(shear_rate), Uoffset=0.0, omega=float(omega), by=by, bz=bz,
                   mhd=True, **kw)

    # -- operators -------------------------------------------------------------
    def _wavenumbers(self, ky, kz):
        ky = torch.as_tensor(ky, dtype=torch.float64, device=self.device)
        kz = torch.as_tensor(kz, dtype=torch.float64, device=self.device)
        ky, kz = torch.broadcast_tensors(ky, kz)
        if bool(((ky * ky + kz * kz) <= 0.0).any()):
            raise ValueError("at least one of ky or kz must be non-zero")
        return ky.reshape(-1), kz.reshape(-1), ky.shape

    def _collocation_batch(self, ky, kz):
        """MHD descriptor pencil (B, 8 nx, 8 nx): blocks (u_x, u_y, u_z, p,
        b_x, b_y, b_z, phi) of collocation values, momentum with the Lorentz
        force of the imposed field, induction with the shear of b_x into b_y,
        continuity and div b = 0 through the multipliers p and phi, the wall
        rows of the velocity (no slip) and of the chosen magnetic condition
        (pcf_linear_jax.py:204-348)."""
        c, n = self._c, self.nx
        B = ky.numel()
        cx = lambda v: v.to(torch.complex128)[:, None, None]  # noqa: E731
        iky, ikz = 1j * cx(ky), 1j * cx(kz)
        k2 = cx(ky * ky + kz * kz)
        I = torch.eye(n, dtype=torch.complex128, device=self.device)
        D, D2 = c["D"], c["D2"]
        U = torch.diag(self.Uoffset + self.Uprime * c["x"])
        lap = D2 - k2 * I
        adv = -iky * U
        ikB = 1j * cx(ky * self.by + kz * self.bz)
        L = torch.zeros(B, 8 * n, 8 * n, dtype=torch.complex128, device=self.device)
        M = torch.zeros_like(L)

        def blk(A, r, col, v):
            A[:, r * n:(r + 1) * n, col * n:(col + 1) * n] += v

        for f in range(3):
            blk(L, f, f, adv + self.nu * lap)
            blk(M, f, f, I)
            blk(L, f, 4 + f, ikB * I)            # Lorentz force of the imposed field
            blk(L, 4 + f, f, ikB * I)            # induction by the imposed field
            blk(L, 4 + f, 4 + f, adv + self.eta * lap)
            blk(M, 4 + f, 4 + f, I)
        blk(L, 0, 3, -D)
        blk(L, 1, 3, -iky * I)
        blk(L, 2, 3, -ikz * I)
        blk(L, 1, 0, (-self.Uprime - 2.0 * self.omega) * I)
        blk(L, 0, 1, 2.0 * self.omega * I)
        blk(L, 3, 0, D)
        blk(L, 3, 1, iky * I)
        blk(L, 3, 2, ikz * I)
        blk(L, 5, 4, self.Uprime * I)
        blk(L, 4, 7, -D)
        blk(L, 5, 7, -iky * I)
        blk(L, 6, 7, -ikz * I)
        blk(L, 7, 4, D)
        blk(L, 7, 5, iky * I)
        blk(L, 7, 6, ikz * I)
        walls = (0, n - 1)
        rows = [f * n + wl for f in range(3) for wl in walls]
        bc = self.magnetic_bc
        # the field's wall rows; pseudo_vacuum and insulating also pin phi
        # there (div b = 0 at the wall follows from their other rows)
        pinned = (4, 5, 6) if bc in ("dirichlet", "conducting") else (4, 5, 6, 7)
        rows += [f * n + wl for f in pinned for wl in walls]
        L[:, rows, :] = 0.0
        M[:, rows, :] = 0.0
        for f in range(3):
            for wl in walls:
                L[:, f * n + wl, f * n + wl] = 1.0
        bx, byb, bzb, phi = 4 * n, 5 * n, 6 * n, 7 * n
        if bc == "dirichlet":
            for b0 in (bx, byb, bzb):
                for wl in walls:
                    L[:, b0 + wl, b0 + wl] = 1.0
        elif bc == "conducting":
            for wl in walls:
                L[:, bx + wl, bx + wl] = 1.0
                L[:, byb + wl, byb:byb + n] = D[wl]
                L[:, bzb + wl, bzb:bzb + n] = D[wl]
        elif bc == "pseudo_vacuum":
            for wl in walls:
                L[:, phi + wl, phi + wl] = 1.0
                L[:, bx + wl, bx:bx + n] = D[wl]
                L[:, byb + wl, byb + wl] = 1.0
                L[:, bzb + wl, bzb + wl] = 1.0
        else:  # insulating: exterior potential field exp(-k |x|) matched at each wall
            k = torch.sqrt(ky * ky + kz * kz).to(torch.complex128)
            for wl, sgn in ((0, 1.0), (n - 1, -1.0)):
                L[:, phi + wl, phi + wl] = 1.0
                L[:, bx + wl, bx:bx + n] = D[wl]
                L[:, bx + wl, bx + wl] += sgn * k
                L[:, byb + wl, byb + wl] = 1.0
                L[:, byb + wl, bx + wl] = sgn * 1j * ky.to(torch.complex128) / k
                L[:, bzb + wl, bzb + wl] = 1.0
                L[:, bzb + wl, bx + wl] = sgn * 1j * kz.to(torch.complex128) / k
        return L, M

    def assemble_batch(self, ky, kz):
        """(L, M) of shape (B, n, n) for the flattened broadcast of ky, kz."""
        ky, kz, _ = self._wavenumbers(ky, kz)
        if self.mhd:
            return self._collocation_batch(ky, kz)
        m, nB = self._m, self.nB
        c = lambda v: v.to(torch.complex128)[:, None, None]  # noqa: E731
        k2 = c(ky * ky + kz * kz)
        iky, ikz = 1j * c(ky), 1j * c(kz)
        lap_u = -m["A1"] - k2 * m["A0"]                       # (phi_i, lap phi_j)
        B = ky.numel()
        L = torch.zeros(B, self.n, self.n, dtype=torch.complex128, device=self.device)
        M = torch.zeros_like(L)
        M[:, :nB, :nB] = lap_u
        M[:, nB:, nB:] = m["B0"]
        L[:, :nB, :nB] = (self.nu * (m["A2"] + 2.0 * k2 * m["A1"] + k2 * k2 * m["A0"])
                          - iky * (self.Uprime * (m["XD2"] - k2 * m["X0"]) + self.Uoffset * lap_u))
        L[:, :nB, nB:] = -2.0 * self.omega * ikz * m["C"].T
        L[:, nB:, :nB] = (self.Uprime + 2.0 * self.omega) * ikz * m["C"]
        L[:, nB:, nB:] = (self.nu * (-m["B1"] - k2 * m["B0"])
                          - iky * (self.Uprime * m["XB"] + self.Uoffset * m["B0"]))
        return L, M

    def assemble(self, ky, kz):
        """(L, M), each (n, n), of one mode (pcf_linear_jax.py:292-348)."""
        L, M = self.assemble_batch(float(ky), float(kz))
        return L[0], M[0]

    def energy_matrix_batch(self, ky, kz, kind="total"):
        """Energy metric Q (B, n, n).  Hydrodynamic operator: q^H Q q =
        int |u_x|^2 + |u_y|^2 + |u_z|^2 dx for the coefficients q = [u; g];
        MHD operator: Clenshaw-Curtis weights on the velocity ("kinetic"),
        field ("magnetic") or both ("total") blocks."""
        if kind not in ("total", "kinetic", "magnetic"):
            raise ValueError("kind must be 'total', 'kinetic', or 'magnetic'")
        if kind == "magnetic" and not self.mhd:
            raise ValueError("magnetic energy norm requires mhd=True")
        ky, kz, _ = self._wavenumbers(ky, kz)
        if self.mhd:  # Clenshaw-Curtis weights on the velocity and/or field blocks
            n = self.nx
            Q = torch.zeros(self.n, self.n, dtype=torch.complex128, device=self.device)
            blocks = ([0, 1, 2] if kind != "magnetic" else []) + ([4, 5, 6] if kind != "kinetic" else [])
            for f in blocks:
                Q[f * n:(f + 1) * n, f * n:(f + 1) * n] = torch.diag(self._c["w"])
            return Q.expand(ky.numel(), self.n, self.n)
        k2 = (ky * ky + kz * kz).to(torch.complex128)[:, None, None]
        m, nB = self._m, self.nB
        Q = torch.zeros(ky.numel(), self.n, self.n, dtype=torch.complex128, device=self.device)
        Q[:, :nB, :nB] = m["A0"] + m["A1"] / k2
        Q[:, nB:, nB:] = m["B0"] / k2
        return Q

    def energy_matrix(self, kind="total", *, ky, kz):
        """The metric of one mode (pcf_linear_jax.py:350-373; here it
        depends on the wavenumber, through u_y, u_z = f(u, g))."""
        return self.energy_matrix_batch(float(ky), float(kz), kind)[0]

    def _operator(self, ky, kz):
        L, M = self.assemble_batch(ky, kz)
        return torch.linalg.solve(M, L)

    # -- modal analysis ----------------------------------------------------------
    def eigs(self, ky, kz, n_return=8, finite_cap=NONMODAL_FINITE_CAP):
        """Growth-sorted eigenpairs with energy (pcf_linear_jax.py:375-379)."""
        L, M = self.assemble(ky, kz)
        w, V = _pencil_eig(L, M)
        w, V = _keep_finite(w, V, finite_cap)
        o = _growth_sort(w)
        w, V = w[o], V[:, o]
        Q = self.energy_matrix("total", ky=ky, kz=kz)
        scale = float(torch.linalg.matrix_norm(Q, ord=2))
        energy = torch.einsum("im,im->m", V.conj(), Q @ V).real
        keep = torch.nonzero(energy > math.sqrt(np.finfo(float).eps) * scale
                             * (V.abs() ** 2).sum(0)).flatten()
        w, V = w[keep], V[:, keep]
        if n_return is not None:
            w, V = w[:n_return], V[:, :n_return]
        return w, V

    def growth_rate(self, ky, kz) -> float:
        """Real part of the leading eigenvalue (pcf_linear_jax.py:381-383)."""
        return float(self.growth_rates(float(ky), float(kz)).reshape(-1)[0])

    def growth_rates(self, ky, kz, finite_cap=NONMODAL_FINITE_CAP) -> torch.Tensor:
        """Leading growth rate of every mode of the broadcast (ky, kz) grid,
        one batched solve and eigenvalue call; shape of the broadcast."""
        _, _, shape = self._wavenumbers(ky, kz)
        w, V = _pencil_eig(*self.assemble_batch(ky, kz), vectors=self.mhd)
        ok = torch.isfinite(w.real) & torch.isfinite(w.imag) & (w.abs() < finite_cap)
        if self.mhd:
            # descriptor pencil: only eigenvectors with energy are modes
            # (multiplier directions carry none), as in ``eigs``
            Q = self.energy_matrix_batch(ky, kz)
            scale = torch.linalg.matrix_norm(Q[:1], ord=2).reshape(())
            energy = torch.einsum("bim,bim->bm", V.conj(), Q @ V).real
            ok &= energy > math.sqrt(np.finfo(float).eps) * scale * (V.abs() ** 2).sum(1)
        re = torch.where(ok, w.real, torch.full_like(w.real, -math.inf))
        return re.max(dim=-1).values.reshape(shape)

    # -- non-modal growth ----------------------------------------------------------
    def optimal_growth(self, ky, kz, times) -> torch.Tensor:
        """G(t) = max_q |q(t)|_E^2 / |q(0)|_E^2 for every mode of the
        broadcast (ky, kz) and every time: G = || R exp(A t) R^-1 ||_2^2,
        A = M^-1 L, Q = R^H R; one batched matrix exponential over
        (mode, time).  Shape (*broadcast, T)."""
        _, _, shape = self._wavenumbers(ky, kz)
        if self.mhd:  # descriptor pencil: the modal route, one mode at a time
            kyf, kzf, _ = self._wavenumbers(ky, kz)
            t = parse_times(times)
            G = [[r["gain"] for r in self.nonmodal_growth(float(a), float(b), t)]
                 for a, b in zip(kyf.tolist(), kzf.tolist(), strict=True)]
            return torch.tensor(G, dtype=torch.float64, device=self.device).reshape(*shape, len(t))
        tt = torch.as_tensor(parse_times(times), dtype=torch.float64, device=self.device)
        A = self._operator(ky, kz)                                            # (B, n, n)
        R = torch.linalg.cholesky(self.energy_matrix_batch(ky, kz)).mH        # Q = R^H R
        E = torch.linalg.matrix_exp(A[:, None] * tt.to(A.dtype)[None, :, None, None])
        P = torch.linalg.solve_triangular(R[:, None], R[:, None] @ E, upper=True, left=False)
        return (torch.linalg.svdvals(P)[..., 0] ** 2).reshape(*shape, tt.numel())

    def nonmodal_growth(self, ky, kz, times, n_modes=None, finite_cap=NONMODAL_FINITE_CAP,
                        energy="total"):
        """Optimal transient growth rows ``{"t", "gain", "amplification"}``
        (pcf_linear_jax.py:385-396).  Hydrodynamic operator, all modes: the
        propagator of ``optimal_growth``; ``n_modes`` or the MHD operator:
        the leading (all finite) eigenvectors through
        ``transient_growth_from_eigs`` in the ``energy`` norm ("kinetic",
        "magnetic" or "total")."""
        Q = self.energy_matrix(energy, ky=ky, kz=kz)
        t = parse_times(times)
        if n_modes is None and not self.mhd:
            gains = self.optimal_growth(float(ky), float(kz), t).reshape(-1).cpu().numpy()
            return _growth_rows(t, gains)
        w, V = _pencil_eig(*self.assemble(ky, kz))
        w, V = _keep_finite(w, V, finite_cap)
        o = _growth_sort(w)
        if n_modes is not None:
            o = o[: int(n_modes)]
        return transient_growth_from_eigs(w[o], V[:, o], Q, t)


def main(argv=None) -> int:
    """Command line of pcf_linear_jax.py:399-460."""
    import argparse

    p = argparse.ArgumentParser(description="Plane-Couette linear/non-modal analysis (B200)")
    p.add_argument("--nx", type=int, default=64)
    p.add_argument("--Re", type=float, default=400.0)
    p.add_argument("--ky", type=float, default=1.0)
    p.add_argument("--kz", type=float, default=1.0)
    p.add_argument("--nonmodal", action="store_true")
    p.add_argument("--times", type=str, default="1,5,10,20")
    p.add_argument("--n-modes", type=int, default=None)
    p.add_argument("--Rm", type=float, default=None)
    p.add_argument("--mhd", action="store_true")
    p.add_argument("--shearpy", action="store_true")
    p.add_argument("--by", type=float, default=0.0)
    p.add_argument("--bz", type=float, default=0.025)
    p.add_argument("--magnetic-bc", choices=list(_MAGNETIC_BCS), default="conducting")
    p.add_argument("--energy", choices=["total", "kinetic", "magnetic"], default="total")
    a = p.parse_args(argv)
    if a.shearpy:
        solver = PlaneCouetteLinear.shearpy(nx=a.nx, Re=a.Re, Rm=a.Rm or a.Re, by=a.by, bz=a.bz,
                                            magnetic_bc=a.magnetic_bc)
    else:
        solver = PlaneCouetteLinear.couette(nx=a.nx, Re=a.Re, Rm=a.Rm, mhd=a.mhd, by=a.by,
                                            bz=a.bz, magnetic_bc=a.magnetic_bc)
    if a.nonmodal:
        print_transient_growth(solver.nonmodal_growth(a.ky, a.kz, parse_times(a.times),
                                                      n_modes=a.n_modes, energy=a.energy))
    else:
        w, _ = solver.eigs(a.ky, a.kz, n_return=8)
        print_eigenvalues(w)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
