"""NumPy FP64 restatement of the reference KMM plane-Couette step (test oracle).

TEST INFRASTRUCTURE ONLY — imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py``; never by the product package.

Every function cites the reference file:line it restates (paths are relative
to the fnauman/jaxfun project).  Arrays are full complex, C-ordered
``(x, y, z)`` with the wall-normal Chebyshev/Legendre axis first, exactly as
the reference stores them.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

import numpy as np
import scipy.fft as sfft

_WORKERS = -1  # scipy.fft thread count (all host cores)


def set_workers(n: int) -> None:
    """Set the number of host threads scipy.fft may use (-1 = all cores)."""
    global _WORKERS
    _WORKERS = int(n)


# ---------------------------------------------------------------------------
# Small axis helpers
# ---------------------------------------------------------------------------


def _bshape(ndim: int, axis: int, n: int) -> tuple[int, ...]:
    shape = [1] * ndim
    shape[axis] = n
    return tuple(shape)


def _apply_matrix(mat: np.ndarray, x: np.ndarray, axis: int) -> np.ndarray:
    """Contract ``mat`` (n_out, n_in) with ``x`` along ``axis``."""
    xm = np.moveaxis(x, axis, 0)
    out = np.tensordot(mat, xm, axes=([1], [0]))
    return np.moveaxis(out, 0, axis)


# ---------------------------------------------------------------------------
# No-pivot banded LU and substitutions
#   diamatrix.py:394-504 (lu_factor, pivot=False), 1936-1973 (kernel)
#   tpmatrix.py:686-799 (batched forward elimination / back substitution)
# ---------------------------------------------------------------------------


def dense_offsets(a: np.ndarray, tol: int = 1000) -> tuple[int, ...]:
    """Diagonals kept by ``DiaMatrix.from_dense`` (diamatrix.py:159-200)."""
    n, m = a.shape
    max_abs = np.abs(a).max()
    if max_abs == 0:
        return ()
    atol = (np.nextafter(max_abs, max_abs + 1) - max_abs) * tol
    return tuple(
        k for k in range(-(n - 1), m) if np.any(np.abs(np.diagonal(a, k)) > atol)
    )


def band_from_dense(a: np.ndarray, offsets, p: int, q: int) -> np.ndarray:
    """Column-aligned band ``band[p + off, j] = A[j - off, j]`` (batched)."""
    n = a.shape[-1]
    band = np.zeros(a.shape[:-2] + (p + q + 1, n), dtype=a.dtype)
    for off in offsets:
        if -p <= off <= q:
            j = np.arange(max(0, off), min(n, n + off))
            band[..., p + off, j] = a[..., j - off, j]
    return band


def lu_banded_nopivot(band: np.ndarray, p: int, q: int) -> np.ndarray:
    """In-place-style Doolittle banded LU without pivoting, batched over the
    leading axes.  Restates ``_lu_banded_no_pivot_kernel``
    (diamatrix.py:1936-1973): for each column k, the multipliers
    ``A[k+s,k]/A[k,k]`` are stored in the sub-diagonals and the trailing
    rows are updated inside the band."""
    band = band.copy()
    c = p
    n = band.shape[-1]
    for k in range(n):
        pivot = band[..., c, k]
        for s in range(1, p + 1):
            if k + s >= n:
                continue
            f = band[..., c - s, k] / pivot
            band[..., c - s, k] = f
            for u in range(1, q + 1):
                j = k + u
                if j >= n:
                    break
                band[..., c + u - s, j] -= f * band[..., c + u, j]
    return band


@dataclass
class BandedLU:
    """Pruned L/U DIA data in the reference's solver layout.

    ``L[..., d, :]`` is the sub-diagonal ``L_offsets[d]`` and ``U[..., d, :]``
    the diagonal ``U_offsets[d]`` (column-aligned), as produced by
    ``TPMatricesWavenumberSolver.__init__`` (tpmatrix.py:1105-1149)."""

    L: np.ndarray
    U: np.ndarray
    L_offsets: tuple[int, ...]
    U_offsets: tuple[int, ...]
    n: int

    @classmethod
    def factor(cls, a: np.ndarray, offsets=None) -> BandedLU:
        """Factor a (batched) dense square matrix restricted to its DIA offsets."""
        if offsets is None:
            ref = a.reshape((-1,) + a.shape[-2:])
            offsets = sorted({o for m in ref for o in dense_offsets(m)})
        p = max((-o for o in offsets if o < 0), default=0)
        q = max((o for o in offsets if o > 0), default=0)
        n = a.shape[-1]
        band = lu_banded_nopivot(band_from_dense(a, offsets, p, q), p, q)
        axes = tuple(range(band.ndim - 2)) + (band.ndim - 1,)
        L_all = [band[..., p + off, :] for off in range(-p, 0)]
        U_all = [band[..., p + off, :] for off in range(0, q + 1)]
        L_off = tuple(
            off for off, d in zip(range(-p, 0), L_all) if np.any(np.abs(d) > 0)
        )
        U_off = tuple(
            off for off, d in zip(range(0, q + 1), U_all) if np.any(np.abs(d) > 0)
        )
        del axes
        L = (
            np.stack([band[..., p + off, :] for off in L_off], axis=-2)
            if L_off
            else np.zeros(band.shape[:-2] + (0, n))
        )
        U = np.stack([band[..., p + off, :] for off in U_off], axis=-2)
        return cls(L=L, U=U, L_offsets=L_off, U_offsets=U_off, n=n)

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        """Solve ``L U x = rhs``; ``rhs`` has shape ``batch + (n,) + extra``
        where ``batch`` matches the factor batch (or is absent for a single
        factor).  Forward elimination then back substitution, restating
        ``_make_wavenumber_batched_solve`` (tpmatrix.py:686-799)."""
        n = self.n
        batch_nd = self.L.ndim - 2
        extra = rhs.ndim - batch_nd - 1

        def coef(arr: np.ndarray, i: int) -> np.ndarray:
            v = arr[..., i]
            return v.reshape(v.shape + (1,) * extra)

        y = np.array(rhs, dtype=np.result_type(rhs, self.U), copy=True)
        ymv = np.moveaxis(y, batch_nd, 0)  # (n, batch..., extra...)
        for i in range(n):
            acc = 0
            for d, off in enumerate(self.L_offsets):
                s = -off
                if i - s >= 0:
                    acc = acc + coef(self.L[..., d, :], i - s) * ymv[i - s]
            ymv[i] = ymv[i] - acc
        main = self.U_offsets.index(0)
        for i in range(n - 1, -1, -1):
            acc = 0
            for d, off in enumerate(self.U_offsets):
                if off == 0:
                    continue
                if i + off < n:
                    acc = acc + coef(self.U[..., d, :], i + off) * ymv[i + off]
            ymv[i] = (ymv[i] - acc) / coef(self.U[..., main, :], i)
        return y


# ---------------------------------------------------------------------------
# 1-D bases
# ---------------------------------------------------------------------------


class Fourier1D:
    """Complex exponential basis (galerkin/Fourier.py)."""

    is_fourier = True

    def __init__(self, N: int, domain=(0.0, 2.0 * math.pi)):
        assert N % 2 == 0
        self.N = int(N)
        self.num_dofs = self.N
        self.domain = (float(domain[0]), float(domain[1]))
        L = self.domain[1] - self.domain[0]
        ref = 2.0 * math.pi
        # orthogonal.py:411-422 (domain_factor = reference length / true length)
        self.df = 1.0 if abs(L - ref) < 1e-12 else ref / L

    def wavenumbers(self, eliminate_highest_freq: bool = False) -> np.ndarray:
        """FFT-ordered integer wavenumbers (Fourier.py:16-22)."""
        k = np.arange(self.N)
        k = np.where(k < (self.N + 1) // 2, k, k - self.N)
        if eliminate_highest_freq and self.N % 2 == 0:
            k[self.N // 2] = 0
        return k

    def mesh(self, n: int | None = None) -> np.ndarray:
        n = self.N if n is None else n
        return np.linspace(self.domain[0], self.domain[1], n, endpoint=False)

    def backward(self, c: np.ndarray, n: int | None, axis: int) -> np.ndarray:
        """Zero-pad in the middle, then ``ifft(norm='forward')``
        (Fourier.py:128-150)."""
        n = self.N if n is None else n
        m = c.shape[axis]
        if n > m:
            lo = np.take(c, np.arange(m // 2), axis=axis)
            hi = np.take(c, np.arange(m // 2, m), axis=axis)
            zshape = list(c.shape)
            zshape[axis] = n - m
            c = np.concatenate((lo, np.zeros(zshape, dtype=c.dtype), hi), axis=axis)
        return sfft.ifft(c, axis=axis, norm="forward", workers=_WORKERS)

    def _truncate(self, out: np.ndarray, axis: int) -> np.ndarray:
        if out.shape[axis] > self.N:
            idx = self.wavenumbers() % out.shape[axis]
            return np.take(out, idx, axis=axis)
        return out

    def forward(self, u: np.ndarray, axis: int) -> np.ndarray:
        """``fft(norm='forward')`` then index truncation (Fourier.py:169-184)."""
        out = sfft.fft(u, axis=axis, norm="forward", workers=_WORKERS)
        return self._truncate(out, axis)

    def scalar_product(self, u: np.ndarray, axis: int) -> np.ndarray:
        """Fourier.py:152-167."""
        out = sfft.fft(u, axis=axis, norm="forward", workers=_WORKERS)
        out = out * (math.tau / self.df)
        return self._truncate(out, axis)

    def derivative_coeffs(self, c: np.ndarray, k: int, axis: int) -> np.ndarray:
        """``(i m)^k c`` with the Nyquist mode zeroed for odd k
        (Fourier.py:210-223)."""
        if k == 0:
            return c
        m = self.wavenumbers(eliminate_highest_freq=k % 2 == 1)
        fac = (1j * m) ** k
        return fac.reshape(_bshape(c.ndim, axis, self.N)) * c

    def norm_squared(self) -> np.ndarray:
        return np.ones(self.N) * 2.0 * np.pi

    def integration_weights(self, n: int) -> np.ndarray:
        """Uniform weights ``2 pi / n / df`` (orthogonal.py quadrature_weights)."""
        return np.full(n, 2.0 * np.pi / n) / self.df

    def matrix_diag(self, i: int, j: int) -> np.ndarray:
        """Diagonal of the Galerkin matrix (test derivative i, trial j)
        including the ``df**(i+j-1)`` domain scaling (Fourier.py:241-268,
        orthogonal.py:547-596)."""
        k = self.wavenumbers()
        d = (1j * k) ** j * (-1j * k) ** i
        if (i + j) % 2 == 0:
            d = d.real
        return d * 2.0 * np.pi * self.df ** (i + j - 1)


class Chebyshev1D:
    """Chebyshev polynomials of the first kind on Gauss nodes
    (galerkin/Chebyshev.py)."""

    family = "C"
    is_fourier = False

    def __init__(self, N: int, domain=(-1.0, 1.0)):
        self.N = int(N)
        self.num_dofs = self.N
        self.domain = (float(domain[0]), float(domain[1]))
        L = self.domain[1] - self.domain[0]
        self.df = 1.0 if abs(L - 2.0) < 1e-12 else 2.0 / L

    def nodes(self, n: int | None = None) -> np.ndarray:
        """Gauss-Chebyshev nodes ``cos(pi + (2k+1) pi/(2n))`` (Chebyshev.py:159-180)."""
        n = self.N if n is None else n
        return np.cos(np.pi + (2 * np.arange(n) + 1) * np.pi / (2 * n))

    def mesh(self, n: int | None = None) -> np.ndarray:
        X = self.nodes(n)
        a = self.domain[0]
        return a + (X + 1.0) / self.df

    def norm_squared(self) -> np.ndarray:
        h = np.full(self.N, np.pi / 2)
        h[0] = np.pi
        return h

    def backward(self, c: np.ndarray, n: int | None = None, axis: int = 0):
        """``0.5 uh[0] + n idct(uh)`` with ``uh = c (-1)^k`` (Chebyshev.py:263-279)."""
        n = self.N if n is None else n
        m = c.shape[axis]
        if n > m:
            pad = [(0, 0)] * c.ndim
            pad[axis] = (0, n - m)
            c = np.pad(c, pad)
        sign = ((-1.0) ** np.arange(n)).reshape(_bshape(c.ndim, axis, n))
        uh = c * sign
        first = np.take(uh, [0], axis=axis)
        return 0.5 * first + n * sfft.idct(uh, type=2, axis=axis, workers=_WORKERS)

    def forward(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """DCT-II, halve mode 0, ``sign/n``, truncate (Chebyshev.py:281-298)."""
        n = u.shape[axis]
        sign = ((-1.0) ** np.arange(n)).reshape(_bshape(u.ndim, axis, n))
        uh = sfft.dct(u, type=2, axis=axis, workers=_WORKERS)
        uh = np.moveaxis(uh, axis, 0).copy()
        uh[0] = uh[0] / 2
        uh = np.moveaxis(uh, 0, axis)
        uh = uh * sign / n
        return np.take(uh, np.arange(self.N), axis=axis)

    def scalar_product(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """Chebyshev.py:300-317."""
        n = u.shape[axis]
        sign = ((-1.0) ** np.arange(n)).reshape(_bshape(u.ndim, axis, n))
        uh = sfft.dct(u, type=2, axis=axis, workers=_WORKERS)
        uh = uh * np.pi * sign / n / 2 / self.df
        return np.take(uh, np.arange(self.N), axis=axis)

    def derivative_coeffs(self, c: np.ndarray, k: int = 1, axis: int = 0):
        """``chebder`` recurrence, applied k times (Chebyshev.py:319-353)."""
        if k == 0:
            return c
        if k > 1:
            return self.derivative_coeffs(
                self.derivative_coeffs(c, k - 1, axis), 1, axis
            )
        cm = np.moveaxis(c, axis, 0)
        N = cm.shape[0] - 1
        d = np.zeros_like(cm)
        x1 = cm[-1] * N * 2
        if N >= 1:
            d[N - 1] = x1
        x0 = np.zeros_like(cm[0])
        for nn in range(N - 2, -1, -1):
            x2 = 2 * (nn + 1) * cm[nn + 1] + x0
            d[nn] = x2
            x0, x1 = x1, x2
        if N >= 2:
            d[0] = d[0] / 2
        return np.moveaxis(d, 0, axis)

    def integration_weights(self, n: int | None = None) -> np.ndarray:
        """Fejer-I weights on the Gauss nodes (Chebyshev.py:182-208)."""
        n = self.N if n is None else n
        theta = np.pi + (2 * np.arange(n) + 1) * np.pi / (2 * n)
        modes = np.arange(1, n // 2 + 1)
        corr = np.sum(
            2.0
            * np.cos(2.0 * theta[:, None] * modes[None, :])
            / (4.0 * modes[None, :] ** 2 - 1.0),
            axis=1,
        )
        return (2.0 / n) * (1.0 - corr) / self.df

    def boundary_rows(self, derivative: int) -> np.ndarray:
        """Values of ``T_n^{(k)}(-1), T_n^{(k)}(+1)``, shape (2, N)."""
        nn = np.arange(self.N, dtype=float)
        if derivative == 0:
            return np.stack([(-1.0) ** nn, np.ones(self.N)])
        if derivative == 1:
            return np.stack([(-1.0) ** (nn + 1) * nn**2, nn**2])
        raise NotImplementedError

    # --- exact 1-D Galerkin matrices (T_i, T_j^{(k)})_w -------------------
    def derivative_matrix_int(self) -> np.ndarray:
        """Integer matrix of the first-derivative coefficient map."""
        N = self.N
        D = np.zeros((N, N), dtype=np.int64)
        for i in range(N):
            for j in range(i + 1, N, 2):
                D[i, j] = j if i == 0 else 2 * j
        return D

    def galerkin_matrix(self, k: int) -> np.ndarray:
        """``(T_i, d^k T_j / dx^k)_w`` on the reference domain (exact integer
        coefficient powers; Chebyshev.py:21-35, 437-487; k=4 is assembled by
        quadrature in the reference, inner.py:945-960, which is exact)."""
        D = np.eye(self.N, dtype=np.int64)
        D1 = self.derivative_matrix_int()
        for _ in range(k):
            D = D1 @ D
        return self.norm_squared()[:, None] * D.astype(np.float64)


class Legendre1D:
    """Legendre polynomials on Gauss-Legendre nodes (galerkin/Legendre.py,
    orthogonal.py Vandermonde transforms)."""

    family = "L"
    is_fourier = False

    def __init__(self, N: int, domain=(-1.0, 1.0)):
        self.N = int(N)
        self.num_dofs = self.N
        self.domain = (float(domain[0]), float(domain[1]))
        L = self.domain[1] - self.domain[0]
        self.df = 1.0 if abs(L - 2.0) < 1e-12 else 2.0 / L
        self._cache: dict[int, tuple[np.ndarray, np.ndarray, np.ndarray]] = {}

    def _quad(self, n: int):
        if n not in self._cache:
            x, w = np.polynomial.legendre.leggauss(n)
            self._cache[n] = (x, w, self.vandermonde(x))
        return self._cache[n]

    def nodes(self, n: int | None = None) -> np.ndarray:
        return self._quad(self.N if n is None else n)[0]

    def mesh(self, n: int | None = None) -> np.ndarray:
        X = self.nodes(n)
        return self.domain[0] + (X + 1.0) / self.df

    def vandermonde(self, X: np.ndarray) -> np.ndarray:
        """``P_j(X_i)`` by the three-term recurrence (Legendre.py:171-193)."""
        V = np.zeros((X.shape[0], self.N))
        V[:, 0] = 1.0
        if self.N > 1:
            V[:, 1] = X
        for i in range(2, self.N):
            V[:, i] = (V[:, i - 1] * X * (2 * i - 1) - V[:, i - 2] * (i - 1)) / i
        return V

    def norm_squared(self) -> np.ndarray:
        return 2.0 / (2.0 * np.arange(self.N) + 1.0)

    def backward(self, c: np.ndarray, n: int | None = None, axis: int = 0):
        """``V[:, :len(c)] @ c`` (orthogonal.py:121-133, 240-253)."""
        n = self.N if n is None else n
        V = self._quad(n)[2]
        return _apply_matrix(V[:, : c.shape[axis]], c, axis)

    def scalar_product(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """``(u w) @ conj(V)`` (orthogonal.py:318-331)."""
        n = u.shape[axis]
        _, w, V = self._quad(n)
        w = w / self.df
        return _apply_matrix((V * w[:, None]).T, u, axis)

    def forward(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """orthogonal.py:310-316."""
        sp = self.scalar_product(u, axis)
        A = self.norm_squared() / self.df
        return sp / A.reshape(_bshape(u.ndim, axis, self.N))

    def derivative_coeffs(self, c: np.ndarray, k: int = 1, axis: int = 0):
        """``legder`` recurrence (Legendre.py:195-227)."""
        if k == 0:
            return c
        if k > 1:
            return self.derivative_coeffs(
                self.derivative_coeffs(c, k - 1, axis), 1, axis
            )
        cm = np.moveaxis(c, axis, 0)
        N = cm.shape[0] - 1
        d = np.zeros_like(cm)
        x1 = cm[-1] * (2 * N - 1)
        if N >= 1:
            d[N - 1] = x1
        x0 = np.zeros_like(cm[0])
        for nn in range(N - 2, -1, -1):
            x2 = (2 * nn + 1) * cm[nn + 1] + (2 * nn + 1) / (2 * nn + 5) * x0
            d[nn] = x2
            x0, x1 = x1, x2
        return np.moveaxis(d, 0, axis)

    def integration_weights(self, n: int | None = None) -> np.ndarray:
        n = self.N if n is None else n
        return self._quad(n)[1] / self.df

    def boundary_rows(self, derivative: int) -> np.ndarray:
        nn = np.arange(self.N, dtype=float)
        if derivative == 0:
            return np.stack([(-1.0) ** nn, np.ones(self.N)])
        if derivative == 1:
            return np.stack(
                [(-1.0) ** (nn + 1) * nn * (nn + 1) / 2, nn * (nn + 1) / 2]
            )
        raise NotImplementedError

    def derivative_matrix_int(self) -> np.ndarray:
        """``P_j' = sum_{i<j, j-i odd} (2i+1) P_i`` as an integer matrix."""
        N = self.N
        D = np.zeros((N, N), dtype=np.int64)
        for i in range(N):
            for j in range(i + 1, N, 2):
                D[i, j] = 2 * i + 1
        return D

    def galerkin_matrix(self, k: int) -> np.ndarray:
        """``(P_i, d^k P_j / dx^k)`` (Legendre.py:19-33, 229-268; k=4 by exact
        quadrature in the reference)."""
        D = np.eye(self.N, dtype=np.int64)
        D1 = self.derivative_matrix_int()
        for _ in range(k):
            D = D1 @ D
        return self.norm_squared()[:, None] * D.astype(np.float64)


def make_orthogonal(family: str, N: int, domain=(-1.0, 1.0)):
    family = family.upper()
    if family.startswith("C"):
        return Chebyshev1D(N, domain)
    if family.startswith("L"):
        return Legendre1D(N, domain)
    raise ValueError("family must be 'C' or 'L'")


def shen_stencil(family: str, bc: str, N: int) -> np.ndarray:
    """Dense stencil ``S`` (N-w, N) with ``phi_i = sum_s S[i, i+s] P_{i+s}``
    (composite.py:797-864)."""
    n = np.arange(N, dtype=float)
    if bc == "dirichlet":
        st = {0: np.ones(N), 2: -np.ones(N)}
        w = 2
    elif bc == "biharmonic":
        if family == "C":
            st = {0: np.ones(N), 2: 2 * (-n - 2) / (n + 3), 4: (n + 1) / (n + 3)}
        else:
            st = {
                0: np.ones(N),
                2: 2 * (-2 * n - 5) / (2 * n + 7),
                4: (2 * n + 3) / (2 * n + 7),
            }
        w = 4
    else:
        raise ValueError(bc)
    S = np.zeros((N - w, N))
    for s, vals in st.items():
        for i in range(N - w):
            S[i, i + s] = vals[i]
    return S


class Composite1D:
    """Shen composite basis ``phi = S P`` (galerkin/composite.py:140-420)."""

    is_fourier = False

    def __init__(self, orth, bc: str):
        self.orth = orth
        self.bc = bc
        self.N = orth.N
        self.S = shen_stencil(orth.family, bc, orth.N)
        self.num_dofs = self.S.shape[0]
        self.df = orth.df
        self.domain = orth.domain
        # composite.py:395-399: mass = S diag(norm^2/df) S^T, no-pivot LU
        self.mass = (self.S * (orth.norm_squared() / orth.df)[None, :]) @ self.S.T
        self.mass_lu = BandedLU.factor(self.mass)

    def mesh(self, n: int | None = None):
        return self.orth.mesh(n)

    def to_orthogonal(self, a: np.ndarray, axis: int = 0) -> np.ndarray:
        """``a @ S`` (composite.py:282-285)."""
        return _apply_matrix(self.S.T, a, axis)

    def _mass_solve(self, b: np.ndarray, axis: int) -> np.ndarray:
        bm = np.moveaxis(b, axis, 0)
        return np.moveaxis(self.mass_lu.solve(bm), 0, axis)

    def scalar_product(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """composite.py:366-370."""
        return _apply_matrix(self.S, self.orth.scalar_product(u, axis), axis)

    def forward(self, u: np.ndarray, axis: int = 0) -> np.ndarray:
        """``mass.solve(scalar_product(u))`` (composite.py:360-364)."""
        return self._mass_solve(self.scalar_product(u, axis), axis)

    def backward(self, c: np.ndarray, n: int | None = None, axis: int = 0):
        return self.orth.backward(self.to_orthogonal(c, axis), n, axis)

    def project_orthogonal_coeffs(self, a: np.ndarray, axis: int = 0):
        """Mass-weight, stencil, banded mass solve (composite.py:292-298)."""
        w = (self.orth.norm_squared() / self.orth.df).reshape(
            _bshape(a.ndim, axis, self.N)
        )
        rhs = _apply_matrix(self.S, a * w, axis)
        return self._mass_solve(rhs, axis)

    def scalar_product_orthogonal_coeffs(self, a: np.ndarray, axis: int = 0):
        """composite.py:300-305."""
        w = (self.orth.norm_squared() / self.orth.df).reshape(
            _bshape(a.ndim, axis, self.N)
        )
        return _apply_matrix(self.S, a * w, axis)

    def integration_weights(self, n: int | None = None):
        return self.orth.integration_weights(n)

    def boundary_rows(self, derivative: int) -> np.ndarray:
        return self.orth.boundary_rows(derivative) @ self.S.T

    def galerkin_matrix(self, k: int) -> np.ndarray:
        """``S (P_i, P_j^{(k)}) S^T`` times ``df**(k-1)`` (inner.py:935-976,
        composite.py:315-320)."""
        X = self.orth.galerkin_matrix(k) * self.df ** (k - 1)
        return self.S @ X @ self.S.T


# ---------------------------------------------------------------------------
# Tensor-product space (galerkin/tensorproductspace.py)
# ---------------------------------------------------------------------------

_SPECTRAL_ORDER = (1, 2, 0)  # tensorproductspace.py:50-77, spectral P("k")
_PHYSICAL_ORDER = (0, 2, 1)  # physical P(None, "k")


class TensorSpace:
    """``TensorProduct(x_space, Fourier, Fourier)``, optionally padded."""

    def __init__(self, x_space, y_space: Fourier1D, z_space: Fourier1D):
        self.spaces = (x_space, y_space, z_space)
        self.x, self.y, self.z = self.spaces

    @property
    def num_dofs(self) -> tuple[int, int, int]:
        return tuple(s.num_dofs for s in self.spaces)

    def quad_counts(self, padding=(1.0, 1.0, 1.0)) -> tuple[int, int, int]:
        """``max(N, int(pf*N))`` per axis (orthogonal.py:361-373)."""
        return tuple(
            max(s.N, int(pf * s.N)) for s, pf in zip(self.spaces, padding, strict=True)
        )

    def mesh(self, counts=None):
        counts = tuple(s.N for s in self.spaces) if counts is None else counts
        xs = [s.mesh(n) for s, n in zip(self.spaces, counts, strict=True)]
        return (
            xs[0][:, None, None],
            xs[1][None, :, None],
            xs[2][None, None, :],
        )

    def backward(self, c: np.ndarray, counts=None) -> np.ndarray:
        return self.backward_primitive(c, (0, 0, 0), counts)

    def backward_primitive(self, c, k=(0, 0, 0), counts=None) -> np.ndarray:
        """Per-axis ``df**k * backward(derivative_coeffs(c, k))`` in the
        spectral axis order (tensorproductspace.py:553-594)."""
        counts = tuple(s.N for s in self.spaces) if counts is None else counts
        z = c
        for ax in _SPECTRAL_ORDER:
            s = self.spaces[ax]
            if isinstance(s, Fourier1D):
                dz = s.derivative_coeffs(z, k[ax], ax)
                z = s.df ** k[ax] * s.backward(dz, counts[ax], ax)
            else:
                orth = s.orth if isinstance(s, Composite1D) else s
                oc = s.to_orthogonal(z, ax) if isinstance(s, Composite1D) else z
                dz = orth.derivative_coeffs(oc, k[ax], ax)
                z = float(orth.df ** k[ax]) * orth.backward(dz, counts[ax], ax)
        return z

    def forward(self, u: np.ndarray) -> np.ndarray:
        """tensorproductspace.py:529-551 (physical axis order)."""
        z = u
        for ax in _PHYSICAL_ORDER:
            z = self.spaces[ax].forward(z, axis=ax)
        return z

    def scalar_product(self, u: np.ndarray) -> np.ndarray:
        z = u
        for ax in _PHYSICAL_ORDER:
            z = self.spaces[ax].scalar_product(z, axis=ax)
        return z

    def to_orthogonal(self, c: np.ndarray) -> np.ndarray:
        """Only the x axis carries a stencil (tensorproductspace.py:596-616)."""
        if isinstance(self.x, Composite1D):
            return self.x.to_orthogonal(c, 0)
        return c

    def differentiate_orthogonal_coeffs(self, c, k) -> np.ndarray:
        """tensorproductspace.py:638-682."""
        z = c
        for ax in _SPECTRAL_ORDER:
            s = self.spaces[ax]
            if k[ax] == 0:
                continue
            if isinstance(s, Fourier1D):
                z = s.df ** k[ax] * s.derivative_coeffs(z, k[ax], ax)
            else:
                orth = s.orth if isinstance(s, Composite1D) else s
                z = float(orth.df ** k[ax]) * orth.derivative_coeffs(z, k[ax], ax)
        return z

    def project_from_orthogonal(self, c: np.ndarray) -> np.ndarray:
        """Fourier axes are identity projections (tensorproductspace.py:706-728)."""
        if isinstance(self.x, Composite1D):
            return self.x.project_orthogonal_coeffs(c, 0)
        return c

    def scalar_product_from_orthogonal(self, c: np.ndarray) -> np.ndarray:
        """tensorproductspace.py:730-754; Fourier axes multiply by the
        diagonal mass ``2 pi / df``."""
        z = c
        for ax in _SPECTRAL_ORDER:
            s = self.spaces[ax]
            if isinstance(s, Fourier1D):
                z = z * (2.0 * np.pi / s.df)
            elif isinstance(s, Composite1D):
                z = s.scalar_product_orthogonal_coeffs(z, ax)
            else:
                w = (s.norm_squared() / s.df).reshape(_bshape(z.ndim, ax, s.N))
                z = z * w
        return z

    def nyquist_mask(self) -> np.ndarray:
        """True where any Fourier axis sits on its Nyquist mode
        (tensorproductspace.py:276-293)."""
        mask = np.zeros(self.num_dofs, dtype=bool)
        for ax in (1, 2):
            s = self.spaces[ax]
            k = s.wavenumbers()
            m = np.abs(k) == s.N // 2
            mask = mask | m.reshape(_bshape(3, ax, s.N))
        return mask

    def mask_nyquist(self, c: np.ndarray) -> np.ndarray:
        return np.where(self.nyquist_mask(), 0, c)

    def wavenumbers(self):
        """Scaled wavenumbers ``k * df`` broadcast (tensorproductspace.py:253-274)."""
        nx = self.x.num_dofs
        ky = self.y.wavenumbers() * self.y.df
        kz = self.z.wavenumbers() * self.z.df
        return (
            np.zeros((nx, 1, 1)),
            ky.reshape(1, -1, 1).astype(float),
            kz.reshape(1, 1, -1).astype(float),
        )

    def integrate(self, values: np.ndarray) -> complex:
        """inner.py:222-262."""
        w = values
        for ax, s in enumerate(self.spaces):
            wt = s.integration_weights(values.shape[ax])
            w = w * wt.reshape(_bshape(3, ax, values.shape[ax]))
        return np.sum(w)


# ---------------------------------------------------------------------------
# Operators: sums of tensor-product terms and the wavenumber solver
# ---------------------------------------------------------------------------


@dataclass
class TPTerms:
    """``sum_t coef_t  X_t (x) diag(fy_t) (x) diag(fz_t)`` — a TPMatrices."""

    terms: list = field(default_factory=list)

    def __add__(self, other: TPTerms) -> TPTerms:
        return TPTerms(self.terms + other.terms)

    def scale(self, alpha: float) -> TPTerms:
        return TPTerms([(c * alpha, X, fy, fz) for (c, X, fy, fz) in self.terms])

    def __sub__(self, other: TPTerms) -> TPTerms:
        return self + other.scale(-1.0)

    def matvec(self, u: np.ndarray) -> np.ndarray:
        """tpmatrix.py:153-157 summed over terms."""
        out = 0
        for c, X, fy, fz in self.terms:
            r = _apply_matrix(X, u, 0)
            r = r * fy[None, :, None] * fz[None, None, :]
            out = out + r * c
        return out


def laplace_terms(xs: Composite1D, y: Fourier1D, z: Fourier1D) -> TPTerms:
    """``(v, lap u)`` as three tensor-product terms."""
    X0, X2 = xs.galerkin_matrix(0), xs.galerkin_matrix(2)
    My, Mz = y.matrix_diag(0, 0), z.matrix_diag(0, 0)
    Dy, Dz = y.matrix_diag(0, 2), z.matrix_diag(0, 2)
    return TPTerms([(1.0, X2, My, Mz), (1.0, X0, Dy, Mz), (1.0, X0, My, Dz)])


def biharmonic_terms(xs: Composite1D, y: Fourier1D, z: Fourier1D) -> TPTerms:
    """``(v, lap lap u)`` as six tensor-product terms."""
    X0, X2, X4 = xs.galerkin_matrix(0), xs.galerkin_matrix(2), xs.galerkin_matrix(4)
    My, Mz = y.matrix_diag(0, 0), z.matrix_diag(0, 0)
    D2y, D2z = y.matrix_diag(0, 2), z.matrix_diag(0, 2)
    D4y, D4z = y.matrix_diag(0, 4), z.matrix_diag(0, 4)
    return TPTerms(
        [
            (1.0, X4, My, Mz),
            (1.0, X0, D4y, Mz),
            (1.0, X0, My, D4z),
            (2.0, X2, D2y, Mz),
            (2.0, X2, My, D2z),
            (2.0, X0, D2y, D2z),
        ]
    )


def mass_terms(xs: Composite1D, y: Fourier1D, z: Fourier1D) -> TPTerms:
    return TPTerms([(1.0, xs.galerkin_matrix(0), y.matrix_diag(0, 0), z.matrix_diag(0, 0))])


class WavenumberSolver:
    """Per-Fourier-mode banded solver (tpmatrix.py:1034-1357, 1900-2029)."""

    def __init__(self, op: TPTerms):
        self.op = op
        terms = op.terms
        n_P = terms[0][1].shape[0]
        Ny, Nz = terms[0][2].shape[0], terms[0][3].shape[0]
        self.shape = (n_P, Ny, Nz)
        W = np.stack([c * np.outer(fy, fz).ravel() for (c, _, fy, fz) in terms])
        offsets = sorted({o for (_, X, _, _) in terms for o in dense_offsets(X)})
        P = np.stack(
            [band_mask(X, offsets) for (_, X, _, _) in terms]
        )  # (n_terms, n_P, n_P)
        B = np.einsum("tf,tij->fij", W, P)  # (n_F, n_P, n_P)
        self.lu = BandedLU.factor(B, offsets)

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        """Transpose to (n_F, n_P), solve, transpose back (tpmatrix.py:1335-1357)."""
        n_P, Ny, Nz = self.shape
        r2 = np.moveaxis(rhs, 0, -1).reshape(Ny * Nz, n_P)
        x = self.lu.solve(r2)
        return np.moveaxis(x.reshape(Ny, Nz, n_P), -1, 0)


def band_mask(X: np.ndarray, offsets) -> np.ndarray:
    out = np.zeros_like(X)
    n = X.shape[0]
    for off in offsets:
        j = np.arange(max(0, off), min(n, n + off))
        out[j - off, j] = X[j - off, j]
    return out


class OneDSolver:
    """A 1-D DIA system with its no-pivot LU (the KMM mean-flow S00)."""

    def __init__(self, A: np.ndarray):
        self.A = A
        self.lu = BandedLU.factor(A)

    def solve(self, rhs: np.ndarray) -> np.ndarray:
        return self.lu.solve(rhs)


# ---------------------------------------------------------------------------
# KMM solver (examples/channelflow_kmm.py) and plane Couette runner
# (examples/pcf_fluctuations_jax.py)
# ---------------------------------------------------------------------------

IMEXRK3_A = (8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0)  # imex_rk.py:96-125
IMEXRK3_B = (0.0, -17.0 / 60.0, -5.0 / 12.0)
_G222 = (2.0 - 2.0**0.5) / 2.0  # imex_rk.py:175-180
_D222 = 1.0 - 1.0 / (2.0 * _G222)
IMEXRK222_A = ((0.0, 0.0, 0.0), (0.0, _G222, 0.0), (0.0, 1.0 - _G222, _G222))
IMEXRK222_B = ((0.0, 0.0, 0.0), (_G222, 0.0, 0.0), (_D222, 1.0 - _D222, 0.0))
SBDF3_IMPLICIT = 1.0 / (11.0 / 6.0)  # sbdf3.py:11-12


@dataclass(frozen=True)
class KMMState:
    """Coefficient-space state (channelflow_kmm.py:50-101)."""

    u: tuple
    g: np.ndarray
    nonlinear_old: tuple | None = None
    nonlinear_older: tuple | None = None
    solution_old: tuple | None = None
    solution_older: tuple | None = None
    history_steps: float = 0.0
    have_old: float = 0.0  # CNAB2: nonlinear_old holds N(u^(n-1))
    previous_dt: float = 0.0


class KMMOracle:
    """Velocity-vorticity KMM solver (channelflow_kmm.py:104-1308)."""

    def __init__(
        self,
        N=(17, 16, 16),
        domain=((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi)),
        nu=1.0 / 600.0,
        dt=0.01,
        family="C",
        padding_factor=(1.0, 1.5, 1.5),
        time_integrator="SBDF3",
        nonlinear_form="rotational",
        coefficient_path="optimized",
    ):
        self.N = tuple(int(n) for n in N)
        self.domain = domain
        self.nu = float(nu)
        self.dt = float(dt)
        self.family = family.upper()[0]
        self.padding_factor = tuple(float(p) for p in padding_factor)
        if time_integrator not in ("SBDF3", "IMEXRK3", "IMEXRK222", "CNAB2"):
            raise ValueError(time_integrator)
        self.time_integrator = time_integrator
        self.nonlinear_form = nonlinear_form
        self.coefficient_path = coefficient_path
        orth = make_orthogonal(self.family, self.N[0], domain[0])
        self.C0 = orth
        self.B0 = Composite1D(orth, "biharmonic")
        self.D0 = Composite1D(orth, "dirichlet")
        self.F1 = Fourier1D(self.N[1], domain[1])
        self.F2 = Fourier1D(self.N[2], domain[2])
        self.TB = TensorSpace(self.B0, self.F1, self.F2)
        self.TD = TensorSpace(self.D0, self.F1, self.F2)
        self.TC = TensorSpace(orth, self.F1, self.F2)
        self.pad_counts = self.TD.quad_counts(self.padding_factor)
        self.counts = tuple(s.N for s in self.TD.spaces)
        self.K = self.TD.wavenumbers()
        k2 = self.K[1] ** 2 + self.K[2] ** 2
        denom = np.where(k2 == 0, 1, k2)
        self.K_over_K2 = (self.K[1] / denom, self.K[2] / denom)  # tpspace:80-99
        self.X = self.TD.mesh()
        self.Xp = self.TD.mesh(self.pad_counts)
        self._build_operators()

    # -- operators (channelflow_kmm.py:261-409) ----------------------------
    def _build_operators(self):
        TBs, TDs = (self.B0, self.F1, self.F2), (self.D0, self.F1, self.F2)
        nu = self.nu
        self.Mu = laplace_terms(*TBs)
        self.Lu = biharmonic_terms(*TBs).scale(nu)
        self.Mg = mass_terms(*TDs)
        self.Lg = laplace_terms(*TDs).scale(nu)
        self.M00 = self.D0.galerkin_matrix(0)
        self.L00 = nu * self.D0.galerkin_matrix(2)

        def factors(gamma):
            return (
                WavenumberSolver(self.Mu - self.Lu.scale(gamma)),
                WavenumberSolver(self.Mg - self.Lg.scale(gamma)),
                OneDSolver(self.M00 - gamma * self.L00),
            )

        if self.time_integrator == "SBDF3":
            self.steady = factors(self.dt * SBDF3_IMPLICIT)
            self.startup = [
                factors((IMEXRK3_A[rk] + IMEXRK3_B[rk]) * self.dt / 2.0)
                for rk in range(3)
            ]
        elif self.time_integrator == "IMEXRK3":
            self.startup = [
                factors((IMEXRK3_A[rk] + IMEXRK3_B[rk]) * self.dt / 2.0)
                for rk in range(3)
            ]
        elif self.time_integrator == "CNAB2":
            self.steady = factors(0.5 * self.dt)  # channelflow_kmm.py:267-274
        else:
            self.steady = factors(self.dt * IMEXRK222_A[1][1])

    # -- transforms of the state -------------------------------------------
    def backward_velocity(self, u, padded=False):
        counts = self.pad_counts if padded else self.counts
        return (
            self.TB.backward(u[0], counts),
            self.TD.backward(u[1], counts),
            self.TD.backward(u[2], counts),
        )

    def state_from_physical(self, u_phys) -> KMMState:
        """channelflow_kmm.py:677-683."""
        u0 = self.TB.mask_nyquist(self.TB.forward(u_phys[0]))
        u1 = self.TD.mask_nyquist(self.TD.forward(u_phys[1]))
        u2 = self.TD.mask_nyquist(self.TD.forward(u_phys[2]))
        g = self.TD.mask_nyquist(1j * self.K[1] * u2 - 1j * self.K[2] * u1)
        return self._reset_history(KMMState(u=(u0, u1, u2), g=g))

    def _reset_history(self, state: KMMState) -> KMMState:
        p = self.primary(state)
        zero = tuple(np.zeros_like(a) for a in p)
        return replace(
            state,
            nonlinear_old=zero,
            nonlinear_older=zero,
            solution_old=zero,
            solution_older=zero,
            history_steps=0.0,
        )

    @staticmethod
    def primary(state: KMMState):
        """channelflow_kmm.py:655-661."""
        return (
            state.u[0],
            state.g,
            np.real(state.u[1][:, 0, 0]),
            np.real(state.u[2][:, 0, 0]),
        )

    def mass_rows(self, p):
        return (
            self.Mu.matvec(p[0]),
            self.Mg.matvec(p[1]),
            self.M00 @ p[2],
            self.M00 @ p[3],
        )

    # -- nonlinear terms -------------------------------------------------
    def base_rotational(self, up, omega):
        return up, omega

    def base_convection(self, n, up, grads):
        return n

    def vorticity_physical(self, u, padded=True):
        """channelflow_kmm.py:699-714."""
        counts = self.pad_counts if padded else self.counts
        sp = (self.TB, self.TD, self.TD)

        def d(c, order):
            return sp[c].backward_primitive(u[c], order, counts)

        return (
            d(2, (0, 1, 0)) - d(1, (0, 0, 1)),
            d(0, (0, 0, 1)) - d(2, (1, 0, 0)),
            d(1, (1, 0, 0)) - d(0, (0, 1, 0)),
        )

    def velocity_gradients(self, u):
        """channelflow_kmm.py:716-740."""
        c = self.pad_counts
        TB, TD = self.TB, self.TD
        return {
            "dudx": TB.backward_primitive(u[0], (1, 0, 0), c),
            "dudy": TB.backward_primitive(u[0], (0, 1, 0), c),
            "dudz": TB.backward_primitive(u[0], (0, 0, 1), c),
            "dvdx": TD.backward_primitive(u[1], (1, 0, 0), c),
            "dvdy": TD.backward_primitive(u[1], (0, 1, 0), c),
            "dvdz": TD.backward_primitive(u[1], (0, 0, 1), c),
            "dwdx": TD.backward_primitive(u[2], (1, 0, 0), c),
            "dwdy": TD.backward_primitive(u[2], (0, 1, 0), c),
            "dwdz": TD.backward_primitive(u[2], (0, 0, 1), c),
        }

    def convection_physical(self, u):
        """channelflow_kmm.py:754-770 (and nonlinear.py:17-29 cross)."""
        up = self.backward_velocity(u, padded=True)
        if self.nonlinear_form == "rotational":
            om = self.vorticity_physical(u)
            a, b = self.base_rotational(up, om)
            cross = (
                a[1] * b[2] - a[2] * b[1],
                a[2] * b[0] - a[0] * b[2],
                a[0] * b[1] - a[1] * b[0],
            )
            return tuple(-v for v in cross)
        g = self.velocity_gradients(u)
        n = (
            up[0] * g["dudx"] + up[1] * g["dudy"] + up[2] * g["dudz"],
            up[0] * g["dvdx"] + up[1] * g["dvdy"] + up[2] * g["dvdz"],
            up[0] * g["dwdx"] + up[1] * g["dwdy"] + up[2] * g["dwdz"],
        )
        return self.base_convection(n, up, g)

    def convection(self, u):
        """channelflow_kmm.py:772-782."""
        n = self.convection_physical(u)
        return tuple(self.TD.mask_nyquist(self.TD.forward(v)) for v in n)

    def nonlinear_rhs(self, H):
        """channelflow_kmm.py:784-829 (transform or coefficient path)."""
        TD, TB = self.TD, self.TB
        if self.coefficient_path == "transform":
            c = self.counts
            Hu = (
                TD.backward_primitive(H[1], (1, 1, 0), c)
                + TD.backward_primitive(H[2], (1, 0, 1), c)
                - TD.backward_primitive(H[0], (0, 2, 0), c)
                - TD.backward_primitive(H[0], (0, 0, 2), c)
            )
            Hg = TD.backward_primitive(H[1], (0, 0, 1), c) - TD.backward_primitive(
                H[2], (0, 1, 0), c
            )
            Nu = TB.scalar_product(Hu)
            Ng = TD.scalar_product(Hg)
        else:
            Ho = tuple(TD.to_orthogonal(h) for h in H)
            doc = TD.differentiate_orthogonal_coeffs
            Hu = (
                doc(Ho[1], (1, 1, 0))
                + doc(Ho[2], (1, 0, 1))
                - doc(Ho[0], (0, 2, 0))
                - doc(Ho[0], (0, 0, 2))
            )
            Hg = doc(Ho[1], (0, 0, 1)) - doc(Ho[2], (0, 1, 0))
            Nu = TB.scalar_product_from_orthogonal(Hu)
            Ng = TD.scalar_product_from_orthogonal(Hg)
        Nv00 = -(self.M00 @ np.real(H[1][:, 0, 0]))
        Nw00 = -(self.M00 @ np.real(H[2][:, 0, 0]))
        return Nu, Ng, np.real(Nv00), np.real(Nw00)

    def reconstruct(self, u0, g, v00, w00):
        """channelflow_kmm.py:831-870."""
        if self.coefficient_path == "transform":
            dudx = self.TB.backward_primitive(u0, (1, 0, 0), self.counts)
            f = self.TD.forward(dudx)
        else:
            do = self.TB.differentiate_orthogonal_coeffs(
                self.TB.to_orthogonal(u0), (1, 0, 0)
            )
            f = self.TD.project_from_orthogonal(do)
        u1 = 1j * (self.K_over_K2[0] * f + self.K_over_K2[1] * g)
        u2 = 1j * (self.K_over_K2[1] * f - self.K_over_K2[0] * g)
        u1[:, 0, 0] = np.real(v00)
        u2[:, 0, 0] = np.real(w00)
        return (
            self.TB.mask_nyquist(u0),
            self.TD.mask_nyquist(u1),
            self.TD.mask_nyquist(u2),
        )

    def _solve_all(self, facs, rhs_u, rhs_g, rhs_v, rhs_w):
        su, sg, s00 = facs
        u0 = su.solve(self.TB.mask_nyquist(rhs_u))
        g = self.TD.mask_nyquist(sg.solve(self.TD.mask_nyquist(rhs_g)))
        means = np.real(s00.solve(np.stack((rhs_v, rhs_w), axis=1)))
        return u0, g, means[:, 0], means[:, 1]

    # -- integrators -----------------------------------------------------
    def step_imexrk3(self, state: KMMState, factors) -> KMMState:
        """channelflow_kmm.py:872-935."""
        dt = self.dt
        u_stage, g_stage = state.u, state.g
        prev = (
            np.zeros_like(state.u[0]),
            np.zeros_like(state.g),
            np.zeros(state.u[1].shape[0]),
            np.zeros(state.u[2].shape[0]),
        )
        for rk in range(3):
            cur = self.nonlinear_rhs(self.convection(u_stage))
            a, b = IMEXRK3_A[rk], IMEXRK3_B[rk]
            gamma = (a + b) * dt / 2.0
            v = np.real(u_stage[1][:, 0, 0])
            w = np.real(u_stage[2][:, 0, 0])
            rhs_u = self.Mu.matvec(u_stage[0]) + gamma * self.Lu.matvec(u_stage[0])
            rhs_g = self.Mg.matvec(g_stage) + gamma * self.Lg.matvec(g_stage)
            rhs_v = self.M00 @ v + gamma * (self.L00 @ v)
            rhs_w = self.M00 @ w + gamma * (self.L00 @ w)
            rhs_u = rhs_u + dt * (a * cur[0] + b * prev[0])
            rhs_g = rhs_g + dt * (a * cur[1] + b * prev[1])
            rhs_v = rhs_v + dt * (a * cur[2] + b * prev[2])
            rhs_w = rhs_w + dt * (a * cur[3] + b * prev[3])
            u0, g, v00, w00 = self._solve_all(factors[rk], rhs_u, rhs_g, rhs_v, rhs_w)
            u_stage = self.reconstruct(u0, g, v00, w00)
            g_stage = g
            prev = cur
        return replace(state, u=u_stage, g=g_stage)

    def step_sbdf3(self, state: KMMState) -> KMMState:
        """channelflow_kmm.py:937-1064 (IMEXRK3 startup, then steady SBDF3)."""
        dt = self.dt
        cur_p = self.primary(state)
        cur_n = self.nonlinear_rhs(self.convection(state.u))
        if state.history_steps < 2:
            adv = self.step_imexrk3(state, self.startup)
        else:
            m0 = self.mass_rows(cur_p)
            m1 = self.mass_rows(state.solution_old)
            m2 = self.mass_rows(state.solution_older)
            rhs = []
            for a0, a1, a2, n0, n1, n2 in zip(
                m0, m1, m2, cur_n, state.nonlinear_old, state.nonlinear_older,
                strict=True,
            ):
                mass = (18.0 * a0 - 9.0 * a1 + 2.0 * a2) / 11.0  # sbdf3.py:15-41
                nl = (18.0 * n0 - 18.0 * n1 + 6.0 * n2) / 11.0
                rhs.append(mass + dt * nl)
            u0, g, v00, w00 = self._solve_all(self.steady, *rhs)
            adv = replace(state, u=self.reconstruct(u0, g, v00, w00), g=g)
        return replace(
            adv,
            nonlinear_old=cur_n,
            nonlinear_older=state.nonlinear_old,
            solution_old=cur_p,
            solution_older=state.solution_old,
            history_steps=min(2.0, state.history_steps + 1.0),
        )

    def step_imexrk222(self, state: KMMState) -> KMMState:
        """Generic ARS branch of ``KMM.step`` (channelflow_kmm.py:1137-1192,
        integrators/coupled.py:13-44)."""
        dt = self.dt
        a, b = IMEXRK222_A, IMEXRK222_B
        p0 = self.primary(state)
        base = self.mass_rows(p0)
        u_stage, g_stage = state.u, state.g
        nl_hist, lin_hist = [], []
        for rk in range(2):
            nl_hist.append(self.nonlinear_rhs(self.convection(u_stage)))
            if rk > 0:
                v = np.real(u_stage[1][:, 0, 0])
                w = np.real(u_stage[2][:, 0, 0])
                lin_hist.append(
                    (
                        self.Lu.matvec(u_stage[0]),
                        self.Lg.matvec(g_stage),
                        self.L00 @ v,
                        self.L00 @ w,
                    )
                )
            rhs = list(base)
            for j in range(rk + 1):
                rhs = [r + dt * b[rk + 1][j] * n for r, n in zip(rhs, nl_hist[j])]
            for j in range(rk):
                rhs = [
                    r + dt * a[rk + 1][j + 1] * ell
                    for r, ell in zip(rhs, lin_hist[j])
                ]
            u0, g, v00, w00 = self._solve_all(self.steady, *rhs)
            u_stage = self.reconstruct(u0, g, v00, w00)
            g_stage = g
        return replace(state, u=u_stage, g=g_stage)

    def step_cnab2(self, state: KMMState) -> KMMState:
        """channelflow_kmm.py:1071-1121: Crank-Nicolson on the linear terms,
        the nonlinear term extrapolated by ``variable_ab2_extrapolate``
        (integrators/cnab2.py:211-240) with r = dt / previous_dt, or taken
        as is on the first step (have_old = 0)."""
        dt = self.dt
        cur_n = self.nonlinear_rhs(self.convection(state.u))
        if state.have_old and state.nonlinear_old is not None:
            r = dt / state.previous_dt
            ext = tuple((1.0 + 0.5 * r) * c - 0.5 * r * p
                        for c, p in zip(cur_n, state.nonlinear_old, strict=True))
        else:
            ext = cur_n
        p = self.primary(state)
        mass = self.mass_rows(p)
        lin = (self.Lu.matvec(p[0]), self.Lg.matvec(p[1]), self.L00 @ p[2], self.L00 @ p[3])
        rhs = [m + 0.5 * dt * ell + dt * n for m, ell, n in zip(mass, lin, ext, strict=True)]
        u0, g, v00, w00 = self._solve_all(self.steady, *rhs)
        return replace(state, u=self.reconstruct(u0, g, v00, w00), g=g, nonlinear_old=cur_n,
                       have_old=1.0, previous_dt=dt)

    def step(self, state: KMMState) -> KMMState:
        if self.time_integrator == "SBDF3":
            return self.step_sbdf3(state)
        if self.time_integrator == "CNAB2":
            return self.step_cnab2(state)
        if self.time_integrator == "IMEXRK3":
            return self.step_imexrk3(state, self.startup)
        return self.step_imexrk222(state)

    def solve(self, state: KMMState, steps: int) -> KMMState:
        for _ in range(int(steps)):
            state = self.step(state)
        return state

    # -- diagnostics ------------------------------------------------------
    def divergence_l2(self, state: KMMState) -> float:
        """channelflow_kmm.py:1287-1293."""
        divu = (
            self.TB.backward_primitive(state.u[0], (1, 0, 0))
            + self.TD.backward_primitive(state.u[1], (0, 1, 0))
            + self.TD.backward_primitive(state.u[2], (0, 0, 1))
        )
        return float(np.sqrt(np.real(self.TC.integrate(np.conj(divu) * divu))))

    def perturbation_energy(self, state: KMMState) -> float:
        up = self.backward_velocity(state.u)
        tot = 0.0
        for ui, sp in zip(up, (self.TB, self.TD, self.TD), strict=True):
            tot += float(np.real(sp.integrate(np.conj(ui) * ui)))
        return tot


class PlaneCouetteOracle(KMMOracle):
    """Fluctuations about ``U_b = U_wall x`` (pcf_fluctuations_jax.py:29-161)."""

    def __init__(self, N=(17, 16, 16), Re=600.0, U_wall=1.0, dt=0.01,
                 perturbation_amplitude=0.05, **kw):
        self.Re = float(Re)
        self.U_wall = float(U_wall)
        self.perturbation_amplitude = float(perturbation_amplitude)
        super().__init__(N=N, nu=self.U_wall / self.Re, dt=dt, **kw)
        self.Ub = self.U_wall * self.X[0]
        self.Ubp = self.U_wall * self.Xp[0]
        self.dUb_dx = self.U_wall

    def initial_state(self) -> KMMState:
        """pcf_fluctuations_jax.py:77-97."""
        x, y, z = self.X
        amp = self.perturbation_amplitude
        wall = 1.0 - x**2
        Ly = self.domain[1][1] - self.domain[1][0]
        Lz = self.domain[2][1] - self.domain[2][0]
        u0 = amp * wall * np.sin(2 * np.pi * y / Ly) * np.cos(2 * np.pi * z / Lz)
        u1 = amp * wall * np.cos(2 * np.pi * y / Ly) * np.sin(2 * np.pi * z / Lz)
        u2 = amp * wall * np.sin(4 * np.pi * y / Ly) * np.cos(4 * np.pi * z / Lz)
        shape = self.counts
        return self.state_from_physical(
            tuple(np.broadcast_to(v, shape).astype(complex) for v in (u0, u1, u2))
        )

    def base_convection(self, n, up, grads):
        """pcf_fluctuations_jax.py:99-106."""
        n0 = n[0] + self.Ubp * grads["dudy"]
        n1 = n[1] + self.Ubp * grads["dvdy"] + up[0] * self.dUb_dx
        n2 = n[2] + self.Ubp * grads["dwdy"]
        return n0, n1, n2

    def base_rotational(self, up, omega):
        """pcf_fluctuations_jax.py:108-112."""
        return (
            (up[0], up[1] + self.Ubp, up[2]),
            (omega[0], omega[1], omega[2] + self.dUb_dx),
        )

    def _wall_trace(self, coeffs, space: Composite1D, derivative=0):
        rows = space.boundary_rows(derivative) * float(space.df) ** derivative
        wall = np.einsum("wi,ijk->wjk", rows, coeffs)
        out = self.F1.backward(wall, None, 1)
        return self.F2.backward(out, None, 2)

    def diagnostics(self, state: KMMState) -> dict[str, float]:
        """pcf_fluctuations_jax.py:131-161."""
        up = self.backward_velocity(state.u)
        ut = (up[0], up[1] + self.Ub, up[2])
        spaces = (self.TB, self.TD, self.TD)
        ep = et = 0.0
        for ui, uti, sp in zip(up, ut, spaces, strict=True):
            ep += float(np.real(sp.integrate(np.conj(ui) * ui)))
            et += float(np.real(sp.integrate(np.conj(uti) * uti)))
        dvdx = self.TD.backward_primitive(state.u[1], (1, 0, 0))
        vol = (
            (self.domain[0][1] - self.domain[0][0])
            * (self.domain[1][1] - self.domain[1][0])
            * (self.domain[2][1] - self.domain[2][0])
        )
        bounds = np.array([self.domain[0][0], self.domain[0][1]])
        uy = self._wall_trace(state.u[1], self.D0) + self.dUb_dx * bounds[:, None, None]
        sh = self._wall_trace(state.u[1], self.D0, 1) + self.dUb_dx
        return {
            "Epert": ep,
            "Etot": et,
            "divL2": self.divergence_l2(state),
            "u_top": float(np.real(np.mean(uy[1]))),
            "u_bot": float(np.real(np.mean(uy[0]))),
            "wall_shear_top": float(np.real(np.mean(sh[1]))),
            "wall_shear_bot": float(np.real(np.mean(sh[0]))),
            "mean_shear": float(np.real(self.TD.integrate(dvdx + self.dUb_dx))) / vol,
        }


# ---------------------------------------------------------------------------
# MHD: plane Couette with a magnetic vector potential (examples/pcf_mhd_jax.py)
# ---------------------------------------------------------------------------


@dataclass
class MHDState:
    """pcf_mhd_jax.py:34-66: flow state, A in TD^3, and the A histories."""

    flow: KMMState
    A: tuple
    nonlinear_A_old: tuple | None = None
    nonlinear_A_older: tuple | None = None
    A_old: tuple | None = None
    A_older: tuple | None = None


class PlaneCouetteMHDOracle(PlaneCouetteOracle):
    """PlaneCouetteMHDJax (pcf_mhd_jax.py:69-789), conducting walls: A in
    TD^3, B = curl A in (TD, TC, TC), J = curl B in (TC, TD, TD)."""

    def __init__(self, N=(17, 16, 16), Re=600.0, Rm=None, U_wall=1.0, dt=0.01,
                 perturbation_amplitude=0.05, magnetic_amplitude=0.05, **kw):
        self.Rm = float(Re if Rm is None else Rm)
        self.eta = float(U_wall) / self.Rm
        self.magnetic_amplitude = float(magnetic_amplitude)
        super().__init__(N=N, Re=Re, U_wall=U_wall, dt=dt,
                         perturbation_amplitude=perturbation_amplitude, **kw)
        self._build_A_operators()

    # pcf_mhd_jax.py:116-139
    def _build_A_operators(self):
        TDs = (self.D0, self.F1, self.F2)
        self.MA = mass_terms(*TDs)
        self.LA = laplace_terms(*TDs).scale(self.eta)

        def factor(gamma):
            return WavenumberSolver(self.MA - self.LA.scale(gamma))

        if self.time_integrator == "SBDF3":
            self.SA = factor(self.dt * SBDF3_IMPLICIT)
            self.SA_startup = [
                factor((IMEXRK3_A[rk] + IMEXRK3_B[rk]) * self.dt / 2.0) for rk in range(3)
            ]
        elif self.time_integrator == "IMEXRK3":
            self.SA_startup = [
                factor((IMEXRK3_A[rk] + IMEXRK3_B[rk]) * self.dt / 2.0) for rk in range(3)
            ]
        else:
            raise NotImplementedError("MHD oracle: SBDF3 or IMEXRK3")

    @property
    def b_spaces(self):
        return (self.TD, self.TC, self.TC)

    @property
    def j_spaces(self):
        return (self.TC, self.TD, self.TD)

    def _A_mass_rhs(self, A):
        return tuple(self.MA.matvec(a) for a in A)

    def _A_eta_lap(self, A):
        return tuple(self.LA.matvec(a) for a in A)

    def _A_solve(self, solver, rhs):
        return tuple(self.TD.mask_nyquist(solver.solve(self.TD.mask_nyquist(r))) for r in rhs)

    def _curl(self, F, spaces_in, spaces_out):
        """pcf_mhd_jax.py:249-291: projected curl without a physical round trip."""
        FO = tuple(sp.to_orthogonal(f) for sp, f in zip(spaces_in, F, strict=True))
        d = lambda sp, f, k: sp.differentiate_orthogonal_coeffs(f, k)  # noqa: E731
        S = spaces_in
        cx = d(S[2], FO[2], (0, 1, 0)) - d(S[1], FO[1], (0, 0, 1))
        cy = d(S[0], FO[0], (0, 0, 1)) - d(S[2], FO[2], (1, 0, 0))
        cz = d(S[1], FO[1], (1, 0, 0)) - d(S[0], FO[0], (0, 1, 0))
        return tuple(
            sp.mask_nyquist(sp.project_from_orthogonal(c))
            for sp, c in zip(spaces_out, (cx, cy, cz), strict=True)
        )

    def update_B_from_A(self, A):
        return self._curl(A, (self.TD, self.TD, self.TD), self.b_spaces)

    def update_J_from_B(self, B):
        return self._curl(B, self.b_spaces, self.j_spaces)

    def _backward_vec(self, F, spaces, padded):
        counts = self.pad_counts if padded else self.counts
        return tuple(sp.backward(f, counts) for sp, f in zip(spaces, F, strict=True))

    @staticmethod
    def _cross(a, b):
        return (a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0])

    # imposed field and rotation (zero here; PlaneCouetteMRIOracle sets them)
    background_b = (0.0, 0.0, 0.0)
    omega = 0.0

    def mhd_convection(self, state: MHDState):
        """pcf_mhd_jax.py:331-346: H = TD[-(u_t x w_t) - J x B], HA = TD[(u + U_b) x B];
        with pcf_mhd_mri_shearpy_jax.py:149-176, B includes the imposed field
        and H the Coriolis term -2 omega e_z x u."""
        flow = state.flow
        n = self.convection_physical(flow.u)
        up = self.backward_velocity(flow.u, padded=True)
        if self.omega != 0.0:
            n = (n[0] - 2.0 * self.omega * up[1], n[1] + 2.0 * self.omega * up[0], n[2])
        B = self.update_B_from_A(state.A)
        J = self.update_J_from_B(B)
        bp = self._backward_vec(B, self.b_spaces, True)
        bp = tuple(b + b0 for b, b0 in zip(bp, self.background_b, strict=True))
        jp = self._backward_vec(J, self.j_spaces, True)
        lorentz = self._cross(jp, bp)
        n = tuple(ni - li for ni, li in zip(n, lorentz, strict=True))
        H = tuple(self.TD.mask_nyquist(self.TD.forward(v)) for v in n)
        utot = (up[0], up[1] + self.Ubp, up[2])
        emf = self._cross(utot, bp)
        HA = tuple(self.TD.mask_nyquist(self.TD.forward(v)) for v in emf)
        return H, HA

    def initial_state(self) -> MHDState:
        """pcf_mhd_jax.py:232-247."""
        flow = super().initial_state()
        x, y, z = self.X
        amp = self.magnetic_amplitude
        shape = self.counts
        ax = np.zeros(shape)
        if amp != 0.0:
            Ly = self.domain[1][1] - self.domain[1][0]
            Lz = self.domain[2][1] - self.domain[2][0]
            ky, kz = 2.0 * np.pi / Ly, 2.0 * np.pi / Lz
            ax = np.broadcast_to(
                amp * (1.0 - x**2) * (1.0 / kz) * np.sin(ky * y) * np.sin(kz * z), shape)
        A = tuple(self.TD.mask_nyquist(self.TD.forward(np.asarray(a, dtype=complex)))
                  for a in (ax, np.zeros(shape), np.zeros(shape)))
        return self._reset_mhd_history(MHDState(flow=flow, A=A))

    def _reset_mhd_history(self, state: MHDState) -> MHDState:
        zero = tuple(np.zeros_like(a) for a in state.A)
        return replace(state, flow=self._reset_history(state.flow), nonlinear_A_old=zero,
                       nonlinear_A_older=zero, A_old=zero, A_older=zero)

    def step_imexrk3_mhd(self, state: MHDState, factors, SA) -> MHDState:
        """pcf_mhd_jax.py:487-560 (coupled Spalart IMEXRK3)."""
        dt = self.dt
        flow_stage, A_stage = state.flow, state.A
        prev = (np.zeros_like(state.flow.u[0]), np.zeros_like(state.flow.g),
                np.zeros(state.flow.u[1].shape[0]), np.zeros(state.flow.u[2].shape[0]))
        prev_A = tuple(np.zeros_like(a) for a in state.A)
        for rk in range(3):
            H, HA = self.mhd_convection(MHDState(flow=flow_stage, A=A_stage))
            cur = self.nonlinear_rhs(H)
            cur_A = self._A_mass_rhs(HA)
            a, b = IMEXRK3_A[rk], IMEXRK3_B[rk]
            gamma = (a + b) * dt / 2.0
            u_stage, g_stage = flow_stage.u, flow_stage.g
            v = np.real(u_stage[1][:, 0, 0])
            w = np.real(u_stage[2][:, 0, 0])
            rhs_u = self.Mu.matvec(u_stage[0]) + gamma * self.Lu.matvec(u_stage[0])
            rhs_g = self.Mg.matvec(g_stage) + gamma * self.Lg.matvec(g_stage)
            rhs_v = self.M00 @ v + gamma * (self.L00 @ v)
            rhs_w = self.M00 @ w + gamma * (self.L00 @ w)
            rhs_u = rhs_u + dt * (a * cur[0] + b * prev[0])
            rhs_g = rhs_g + dt * (a * cur[1] + b * prev[1])
            rhs_v = rhs_v + dt * (a * cur[2] + b * prev[2])
            rhs_w = rhs_w + dt * (a * cur[3] + b * prev[3])
            mA, lA = self._A_mass_rhs(A_stage), self._A_eta_lap(A_stage)
            rhs_A = [mA[i] + gamma * lA[i] + dt * (a * cur_A[i] + b * prev_A[i]) for i in range(3)]
            u0, g, v00, w00 = self._solve_all(factors[rk], rhs_u, rhs_g, rhs_v, rhs_w)
            flow_stage = replace(flow_stage, u=self.reconstruct(u0, g, v00, w00), g=g)
            A_stage = self._A_solve(SA[rk], rhs_A)
            prev, prev_A = cur, cur_A
        return replace(state, flow=replace(state.flow, u=flow_stage.u, g=flow_stage.g), A=A_stage)

    def step_sbdf3_mhd(self, state: MHDState) -> MHDState:
        """pcf_mhd_jax.py:562-715 (IMEXRK3 startup, then steady SBDF3)."""
        dt = self.dt
        flow = state.flow
        cur_p = self.primary(flow)
        H, HA = self.mhd_convection(state)
        cur_n = self.nonlinear_rhs(H)
        cur_nA = self._A_mass_rhs(HA)
        if flow.history_steps < 2:
            adv = self.step_imexrk3_mhd(state, self.startup, self.SA_startup)
        else:
            def comb(m0, m1, m2, n0, n1, n2):
                return (18.0 * m0 - 9.0 * m1 + 2.0 * m2) / 11.0 + dt * (
                    18.0 * n0 - 18.0 * n1 + 6.0 * n2) / 11.0  # sbdf3.py:15-41
            rhs = [comb(*t) for t in zip(
                self.mass_rows(cur_p), self.mass_rows(flow.solution_old),
                self.mass_rows(flow.solution_older), cur_n, flow.nonlinear_old,
                flow.nonlinear_older, strict=True)]
            rhs_A = [comb(*t) for t in zip(
                self._A_mass_rhs(state.A), self._A_mass_rhs(state.A_old),
                self._A_mass_rhs(state.A_older), cur_nA, state.nonlinear_A_old,
                state.nonlinear_A_older, strict=True)]
            u0, g, v00, w00 = self._solve_all(self.steady, *rhs)
            adv = replace(state, flow=replace(flow, u=self.reconstruct(u0, g, v00, w00), g=g),
                          A=self._A_solve(self.SA, rhs_A))
        new_flow = replace(
            adv.flow, nonlinear_old=cur_n, nonlinear_older=flow.nonlinear_old,
            solution_old=cur_p, solution_older=flow.solution_old,
            history_steps=min(2.0, flow.history_steps + 1.0))
        return replace(adv, flow=new_flow, nonlinear_A_old=cur_nA,
                       nonlinear_A_older=state.nonlinear_A_old, A_old=state.A,
                       A_older=state.A_old)

    def step(self, state: MHDState) -> MHDState:
        if self.time_integrator == "SBDF3":
            return self.step_sbdf3_mhd(state)
        return self.step_imexrk3_mhd(state, self.startup, self.SA_startup)

    def solve(self, state: MHDState, steps: int) -> MHDState:
        for _ in range(int(steps)):
            state = self.step(state)
        return state

    def magnetic_divergence_l2(self, state: MHDState) -> float:
        """pcf_mhd_jax.py:736-744."""
        B = self.update_B_from_A(state.A)
        S = self.b_spaces
        divb = (S[0].backward_primitive(B[0], (1, 0, 0))
                + S[1].backward_primitive(B[1], (0, 1, 0))
                + S[2].backward_primitive(B[2], (0, 0, 1)))
        return float(np.sqrt(np.real(self.TC.integrate(np.conj(divb) * divb))))

    def diagnostics(self, state: MHDState) -> dict[str, float]:
        """pcf_mhd_jax.py:752-765."""
        out = super().diagnostics(state.flow)
        B = self.update_B_from_A(state.A)
        bp = self._backward_vec(B, self.b_spaces, False)
        emag = 0.0
        for bi, sp in zip(bp, self.b_spaces, strict=True):
            emag += float(np.real(sp.integrate(np.conj(bi) * bi)))
        out["divB_L2"] = self.magnetic_divergence_l2(state)
        out["Emag"] = emag
        return out


class PlaneCouetteMRIOracle(PlaneCouetteMHDOracle):
    """PlaneCouetteMRIShearpyJax's dynamics (pcf_mhd_mri_shearpy_jax.py:36-176):
    nu = 1/Re, eta = 1/Rm (U_wall = 1 in the parent), base flow
    U_b = -shear_rate x, Coriolis -2 omega e_z x u, imposed field B0.  The
    initial state is the parent's (tests load their own states)."""

    def __init__(self, N=(17, 16, 16), Re=400.0, Rm=None, omega=1.0, shear_rate=1.0,
                 background_b=(0.0, 0.0, 0.025), dt=0.01, perturbation_amplitude=0.05,
                 magnetic_amplitude=0.0, **kw):
        super().__init__(N=N, Re=Re, Rm=Rm, U_wall=1.0, dt=dt,
                         perturbation_amplitude=perturbation_amplitude,
                         magnetic_amplitude=magnetic_amplitude, **kw)
        self.omega = float(omega)
        self.shear_rate = float(shear_rate)
        self.background_b = tuple(float(v) for v in background_b)
        self.U_wall = -self.shear_rate
        self.Ub = -self.shear_rate * self.X[0]
        self.Ubp = -self.shear_rate * self.Xp[0]
        self.dUb_dx = -self.shear_rate


# ---------------------------------------------------------------------------
# 2-D Helmholtz: -lap u + alpha u = f on Chebyshev-Dirichlet (x) x Fourier (y)
# (la/solvers.py:22-61; the pipeline of the 2-D Helmholtz benchmark case)
# ---------------------------------------------------------------------------


def helmholtz2d_forcing(N=(64, 64), seed=1) -> np.ndarray:
    """Seeded orthogonal-Chebyshev x Fourier coefficients of f:
    (a + i b)/sqrt(2) (1 + j)^-2 (1 + |k|)^-2, a, b ~ N(0, 1) (PCG64), made
    Hermitian in k (a real f) with the Nyquist mode zero."""
    Nx, Ny = N
    rng = np.random.Generator(np.random.PCG64(seed))
    a = rng.standard_normal((Nx, Ny))
    b = rng.standard_normal((Nx, Ny))
    j = np.arange(Nx)[:, None]
    k = np.fft.fftfreq(Ny, 1.0 / Ny)[None, :]
    c = (a + 1j * b) / np.sqrt(2.0) * (1.0 + j) ** -2 * (1.0 + np.abs(k)) ** -2
    c[:, Ny // 2] = 0.0
    kk = (-np.arange(Ny)) % Ny
    return 0.5 * (c + np.conj(c[:, kk]))


def helmholtz2d_solve(f_hat: np.ndarray, domain=((-1.0, 1.0), (0.0, 2.0 * math.pi)),
                      alpha: float = 1.0):
    """Reference FP64 solution: f = TC.backward(f_hat); per Fourier mode the
    Galerkin system (-(phi_i, phi_j'') + (k^2 + alpha)(phi_i, phi_j)) u = (phi_i, f)
    solved densely; returns (Dirichlet x Fourier coefficients, u on the mesh)."""
    Nx, Ny = f_hat.shape
    orth = make_orthogonal("C", Nx, domain[0])
    D = Composite1D(orth, "dirichlet")
    F = Fourier1D(Ny, domain[1])
    f = F.backward(orth.backward(f_hat, None, 0), None, 1)
    rhs = D.scalar_product(F.forward(f, 1), 0)
    G0, G2 = D.galerkin_matrix(0), D.galerkin_matrix(2)
    k = F.wavenumbers() * F.df
    u_hat = np.empty_like(rhs)
    for m in range(Ny):
        u_hat[:, m] = np.linalg.solve(-G2 + (k[m] ** 2 + alpha) * G0, rhs[:, m])
    u = F.backward(D.backward(u_hat, None, 0), None, 1)
    return u_hat, u
