"""NumPy/SciPy restatement of the reference's plane-Couette linear-stability
tools, hydrodynamic and MHD (test oracle).

TEST INFRASTRUCTURE ONLY — imported by ``tests/``; never by the product
package.

Restates:

* ``src/jaxfun/la/eig.py:12-125,145-242`` — growth ordering, finite and
  physical eigensystems of a pencil ``L q = s M q``, optimal transient growth
  from a modal basis in an energy metric;
* ``examples/pcf_linear_jax.py:29-66,69-397`` — the primitive-variable
  (u_x, u_y, u_z, p [, b_x, b_y, b_z, phi]) Chebyshev-Lobatto collocation
  operator of plane Couette flow with base flow ``U(x) = Uoffset + Uprime x``
  along y, a rotation ``omega`` about z and, with ``mhd=True``, an imposed
  field (0, by, bz) and the four magnetic wall conditions; wall conditions
  are rows with zero mass (their eigenvalues lie at infinity and are
  filtered).

Pinned against the reference's recorded outputs of these tools
(``couette/couette_linear_benchmarks.md``, in
``tests/golden/reference_linear_goldens.json``).
"""

from __future__ import annotations

import numpy as np
from scipy.linalg import eig as qz_eig, svdvals

MODAL_FINITE_CAP = 1.0e6      # la/eig.py:8
NONMODAL_FINITE_CAP = 1.0e8   # la/eig.py:9


def growth_order(w: np.ndarray) -> np.ndarray:
    """la/eig.py:12-19: descending real part, then descending imaginary part."""
    w = np.asarray(w)
    if w.size == 0:
        return np.zeros(0, dtype=int)
    return np.lexsort((-w.imag, -w.real))


def parse_times(value) -> np.ndarray:
    """la/eig.py:22-35."""
    if isinstance(value, str):
        items = [s for s in value.replace(";", ",").split(",") if s.strip()]
        times = [float(s) for s in items]
    else:
        times = list(value)
    if not times:
        raise ValueError("at least one time is required")
    out = np.asarray(times, dtype=float)
    if (out < 0).any():
        raise ValueError("non-modal times must be non-negative")
    return out


def finite_eigensystem(L, M, *, finite_cap=NONMODAL_FINITE_CAP, n_return=None):
    """la/eig.py:57-77: QZ eigenpairs, finite and below the cap, growth-sorted."""
    w, V = qz_eig(np.asarray(L), np.asarray(M))
    keep = np.isfinite(w) & (np.abs(w) < finite_cap)
    w, V = w[keep], V[:, keep]
    o = growth_order(w)
    w, V = w[o], V[:, o]
    if n_return is not None:
        w, V = w[:n_return], V[:, :n_return]
    return w, V


def generalized_eig(L, M, *, vectors=False, finite_cap=MODAL_FINITE_CAP, sort=True):
    """la/eig.py:166-194."""
    w, V = qz_eig(np.asarray(L), np.asarray(M))
    keep = np.isfinite(w) & (np.abs(w) < finite_cap)
    w, V = w[keep], V[:, keep]
    if sort and len(w):
        o = growth_order(w)
        w, V = w[o], V[:, o]
    return (w, V) if vectors else w


def physical_eigensystem(L, M, metric, *, finite_cap=NONMODAL_FINITE_CAP, n_return=None,
                         metric_rtol=None):
    """la/eig.py:197-242: drop eigenvectors with (relatively) no energy in
    ``metric`` (threshold sqrt(eps) by default, against the metric's 2-norm
    times the vector's squared Euclidean norm)."""
    tol = float(np.sqrt(np.finfo(float).eps)) if metric_rtol is None else float(metric_rtol)
    if not np.isfinite(tol) or tol < 0.0:
        raise ValueError("metric_rtol must be finite and nonnegative")
    w, V = finite_eigensystem(L, M, finite_cap=finite_cap)
    Q = np.asarray(metric, dtype=complex)
    if Q.shape != (V.shape[0], V.shape[0]):
        raise ValueError(f"energy metric must have shape {(V.shape[0],) * 2}, got {Q.shape}")
    if V.shape[1] == 0:
        return w, V
    scale = float(np.linalg.norm(Q, ord=2))
    if not np.isfinite(scale) or scale <= 0.0:
        raise ValueError("energy metric must have a finite positive scale")
    energy = np.real(np.einsum("im,ij,jm->m", V.conj(), Q, V))
    keep = energy > tol * scale * np.sum(np.abs(V) ** 2, axis=0)
    w, V = w[keep], V[:, keep]
    if n_return is not None:
        w, V = w[:n_return], V[:, :n_return]
    return w, V


def transient_growth_from_eigs(evals, evecs, metric, times, *, metric_rtol=1.0e-10):
    """la/eig.py:80-124: G(t) = || F exp(Lambda t) F^+ ||_2^2 with F the
    square root of the metric restricted to the modal span (directions of
    relatively negligible energy removed)."""
    lam = np.asarray(evals, dtype=complex)
    V = np.asarray(evecs, dtype=complex)
    Q = np.asarray(metric, dtype=complex)
    times = parse_times(times)
    if lam.size == 0 or V.size == 0:
        raise ValueError("no finite eigenvectors available for non-modal growth")
    G = V.conj().T @ Q @ V
    G = 0.5 * (G + G.conj().T)
    d, U = np.linalg.eigh(G)
    big = float(np.max(np.abs(d))) if d.size else 0.0
    keep = d > max(metric_rtol * big, np.finfo(float).eps)
    if not keep.any():
        raise ValueError("energy metric is singular on all retained modes")
    d, U = d[keep], U[:, keep]
    s = np.sqrt(d)
    F = s[:, None] * U.conj().T
    rows = []
    for t in times:
        P = (F @ (np.exp(lam * float(t))[:, None] * U)) / s[None, :]
        g = float(svdvals(P)[0] ** 2)
        rows.append({"t": float(t), "gain": g, "amplification": float(np.sqrt(g))})
    return rows


def cheb_lobatto(n: int):
    """pcf_linear_jax.py:29-66: Chebyshev-Lobatto points x_j = cos(pi j/N)
    (x_0 = +1), the collocation derivative matrices D, D^2 (negative-sum
    diagonal) and the Clenshaw-Curtis weights."""
    n = int(n)
    if n < 4:
        raise ValueError("nx must be at least 4")
    N = n - 1
    j = np.arange(n)
    x = np.cos(np.pi * j / N)
    c = np.where((j == 0) | (j == N), 2.0, 1.0) * (-1.0) ** j
    dx = x[:, None] - x[None, :] + np.eye(n)
    D = np.outer(c, 1.0 / c) / dx
    D = D - np.diag(D.sum(axis=1))
    # Clenshaw-Curtis: w_j = (c_j / N) (1 - sum_k b_k cos(2 k theta_j) / (4k^2 - 1))
    theta = np.pi * j / N
    w = np.empty(n)
    inner = np.ones(n)
    for k in range(1, N // 2 + 1):
        b = 1.0 if 2 * k == N else 2.0
        inner -= b * np.cos(2 * k * theta) / (4.0 * k * k - 1.0)
    w[:] = 2.0 * inner / N
    w[0] = w[-1] = 1.0 / (N * N - 1.0) if N % 2 == 0 else 1.0 / (N * N)
    return x, D, D @ D, w


class PlaneCouetteLinearOracle:
    """pcf_linear_jax.py:69-397: blocks (u_x, u_y, u_z, p) and, with
    ``mhd=True``, (b_x, b_y, b_z, phi) (phi: the multiplier of div b = 0),
    each ``nx`` collocation values."""

    BCS = ("conducting", "dirichlet", "pseudo_vacuum", "insulating")

    def __init__(self, nx=64, nu=1.0e-3, eta=1.0e-3, Uprime=1.0, Uoffset=0.0, omega=0.0,
                 by=0.0, bz=0.0, mhd=False, magnetic_bc="conducting"):
        if magnetic_bc not in self.BCS:
            raise ValueError("magnetic_bc must be 'conducting', 'dirichlet', 'pseudo_vacuum' "
                             "or 'insulating'")
        self.nx, self.nu, self.eta = int(nx), float(nu), float(eta)
        self.Uprime, self.Uoffset, self.omega = float(Uprime), float(Uoffset), float(omega)
        self.by, self.bz, self.mhd, self.magnetic_bc = float(by), float(bz), bool(mhd), magnetic_bc
        self.x, self.D, self.D2, self.weights = cheb_lobatto(self.nx)
        self.nb = 8 if self.mhd else 4

    @classmethod
    def couette(cls, nx=64, Re=400.0, Rm=None, U_wall=1.0, mhd=False, **kw):
        """pcf_linear_jax.py:141-152."""
        Rm = Re if Rm is None else Rm
        return cls(nx=nx, nu=float(U_wall) / float(Re), eta=float(U_wall) / float(Rm),
                   Uprime=float(U_wall), mhd=mhd, **kw)

    @classmethod
    def shearpy(cls, nx=64, Re=1000.0, Rm=1000.0, shear_rate=1.0, omega=2.0 / 3.0, by=0.0,
                bz=0.025, velocity_scale=1.0, **kw):
        """pcf_linear_jax.py:154-178."""
        return cls(nx=nx, nu=float(velocity_scale) / float(Re), eta=float(velocity_scale) / float(Rm),
                   Uprime=-float(shear_rate), omega=float(omega), by=by, bz=bz, mhd=True, **kw)

    def assemble(self, ky, kz):
        """pcf_linear_jax.py:292-348 with the wall rows of
        pcf_linear_jax.py:204-290."""
        ky, kz = float(ky), float(kz)
        k2 = ky * ky + kz * kz
        if k2 <= 0.0:
            raise ValueError("at least one of ky or kz must be non-zero")
        n, nb = self.nx, self.nb
        I = np.eye(n, dtype=complex)
        L = np.zeros((nb * n, nb * n), dtype=complex)
        M = np.zeros_like(L)

        def blk(A, r, c, v):
            A[r * n:(r + 1) * n, c * n:(c + 1) * n] += v

        lap = self.D2 - k2 * I
        adv = -1j * ky * np.diag(self.Uoffset + self.Uprime * self.x)
        for c in range(3):
            blk(L, c, c, adv + self.nu * lap)
            blk(M, c, c, I)
        # pressure gradient, shear and rotation, continuity
        blk(L, 0, 3, -self.D)
        blk(L, 1, 3, -1j * ky * I)
        blk(L, 2, 3, -1j * kz * I)
        blk(L, 1, 0, (-self.Uprime - 2.0 * self.omega) * I)
        blk(L, 0, 1, 2.0 * self.omega * I)
        blk(L, 3, 0, self.D)
        blk(L, 3, 1, 1j * ky * I)
        blk(L, 3, 2, 1j * kz * I)
        if self.mhd:
            # Lorentz force and induction by the imposed field, shear of b_x
            # into b_y, the magnetic multiplier and div b = 0
            ikB = 1j * (ky * self.by + kz * self.bz)
            for c in range(3):
                blk(L, c, 4 + c, ikB * I)
                blk(L, 4 + c, c, ikB * I)
                blk(L, 4 + c, 4 + c, adv + self.eta * lap)
                blk(M, 4 + c, 4 + c, I)
            blk(L, 5, 4, self.Uprime * I)
            blk(L, 4, 7, -self.D)
            blk(L, 5, 7, -1j * ky * I)
            blk(L, 6, 7, -1j * kz * I)
            blk(L, 7, 4, self.D)
            blk(L, 7, 5, 1j * ky * I)
            blk(L, 7, 6, 1j * kz * I)

        def row(r, entries):
            L[r, :] = 0.0
            M[r, :] = 0.0
            for cols, vals in entries:
                L[r, cols] = vals

        walls = (0, n - 1)
        for c in range(3):
            for wall in walls:
                row(c * n + wall, [(c * n + wall, 1.0)])
        if self.mhd:
            bx, by_, bz_, phi = 4 * n, 5 * n, 6 * n, 7 * n
            bc = self.magnetic_bc
            if bc == "insulating":
                k = float(np.hypot(ky, kz))
                for wall, sgn in ((0, 1.0), (n - 1, -1.0)):
                    row(phi + wall, [(phi + wall, 1.0)])
                    robin = self.D[wall, :].astype(complex).copy()
                    robin[wall] += sgn * k
                    row(bx + wall, [(slice(bx, bx + n), robin)])
                    row(by_ + wall, [(by_ + wall, 1.0), (bx + wall, sgn * 1j * ky / k)])
                    row(bz_ + wall, [(bz_ + wall, 1.0), (bx + wall, sgn * 1j * kz / k)])
            elif bc == "dirichlet":
                for b0 in (bx, by_, bz_):
                    for wall in walls:
                        row(b0 + wall, [(b0 + wall, 1.0)])
            elif bc == "pseudo_vacuum":
                for wall in walls:
                    row(phi + wall, [(phi + wall, 1.0)])
                    row(bx + wall, [(slice(bx, bx + n), self.D[wall, :])])
                    row(by_ + wall, [(by_ + wall, 1.0)])
                    row(bz_ + wall, [(bz_ + wall, 1.0)])
            else:  # conducting
                for wall in walls:
                    row(bx + wall, [(bx + wall, 1.0)])
                    row(by_ + wall, [(slice(by_, by_ + n), self.D[wall, :])])
                    row(bz_ + wall, [(slice(bz_, bz_ + n), self.D[wall, :])])
        return L, M

    def energy_matrix(self, kind="total"):
        """pcf_linear_jax.py:350-373."""
        if kind not in ("total", "kinetic", "magnetic"):
            raise ValueError("kind must be 'total', 'kinetic', or 'magnetic'")
        if kind == "magnetic" and not self.mhd:
            raise ValueError("magnetic energy norm requires mhd=True")
        n = self.nx
        Q = np.zeros((self.nb * n, self.nb * n), dtype=complex)
        blocks = []
        if kind in ("total", "kinetic"):
            blocks += [0, 1, 2]
        if self.mhd and kind in ("total", "magnetic"):
            blocks += [4, 5, 6]
        for c in blocks:
            Q[c * n:(c + 1) * n, c * n:(c + 1) * n] = np.diag(self.weights)
        return Q

    def eigs(self, ky, kz, n_return=8, finite_cap=NONMODAL_FINITE_CAP):
        """pcf_linear_jax.py:375-379."""
        L, M = self.assemble(ky, kz)
        return physical_eigensystem(L, M, self.energy_matrix("total"), finite_cap=finite_cap,
                                    n_return=n_return)

    def growth_rate(self, ky, kz):
        """pcf_linear_jax.py:381-383."""
        w, _ = self.eigs(ky, kz, n_return=1)
        return float(w[0].real) if len(w) else float("nan")

    def nonmodal_growth(self, ky, kz, times, n_modes=None, finite_cap=NONMODAL_FINITE_CAP,
                        energy="total"):
        """pcf_linear_jax.py:385-396."""
        w, V = finite_eigensystem(*self.assemble(ky, kz), finite_cap=finite_cap, n_return=n_modes)
        return transient_growth_from_eigs(w, V, self.energy_matrix(energy), times)
