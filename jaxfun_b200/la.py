"""``jaxfun.la`` drop-ins backed by the sm_100a kernels.

Mirrors the reference objects used on the Couette hot path:

* ``DiaMatrix`` (src/jaxfun/la/diamatrix.py:100-348): column-aligned DIA
  storage ``data[d, j] = A[j - offsets[d], j]``, ``matvec(x, axis)``,
  ``rmatvec(x, axis)``, ``lu_factor()`` (no pivoting), ``solve``;
* ``TPMatrix`` / ``TPMatrices`` (src/jaxfun/la/tpmatrix.py:153-157, 300-428):
  sums of Kronecker products applied axis by axis;
* ``tpmats_wavenumber_factor`` / ``TPMatricesWavenumberSolver``
  (tpmatrix.py:1900-2029, 1034-1677): per-Fourier-mode banded LU and the
  batched substitution, with ``solve``, ``solve_many``, ``runtime_args``,
  ``solve_with_runtime_args`` and ``solve_many_with_runtime_args``.

Tensors are torch CUDA tensors (float64 matrices, float64 or complex128
right-hand sides).  Torch is used only to hold and reshape device memory;
every product, factorisation and solve runs in ``libjfb200.so``.
"""

from __future__ import annotations

import ctypes
from collections.abc import Sequence

import torch

from . import _lib


def _stream(t: torch.Tensor) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _require_cuda(*ts: torch.Tensor) -> None:
    for t in ts:
        if not t.is_cuda:
            raise ValueError("jaxfun_b200.la operates on CUDA tensors only")


class SolverNotApplicable(ValueError):
    """Raised when a TPMatrices system is not Fourier x polynomial
    (tpmatrix.py:1955-1960)."""


class DiaMatrix:
    """DIA sparse matrix, scipy.sparse.dia compatible (diamatrix.py:100-157)."""

    def __init__(self, data: torch.Tensor, offsets: Sequence[int], shape: tuple[int, int]):
        data = torch.as_tensor(data, dtype=torch.float64)
        if data.dim() != 2 or data.shape[0] != len(offsets) or data.shape[1] != shape[1]:
            raise ValueError("data must have shape (len(offsets), n_cols)")
        self.data = data.contiguous()
        self.offsets = tuple(int(o) for o in offsets)
        self.shape = (int(shape[0]), int(shape[1]))
        self._lu = None

    @classmethod
    def from_dense(cls, a: torch.Tensor, offsets: Sequence[int] | None = None,
                   tol: int = 100) -> DiaMatrix:
        """Build from a dense matrix, keeping diagonals above ``ulp(max)*tol``
        (diamatrix.py:159-225)."""
        a = torch.as_tensor(a, dtype=torch.float64)
        n, m = a.shape
        if offsets is None:
            mx = a.abs().max().item()
            atol = (torch.nextafter(torch.tensor(mx, dtype=torch.float64),
                                    torch.tensor(mx + 1, dtype=torch.float64)).item() - mx) * tol
            offsets = [k for k in range(-(n - 1), m)
                       if torch.diagonal(a, k).abs().max().item() > atol]
        data = torch.zeros((len(offsets), m), dtype=torch.float64, device=a.device)
        for p, k in enumerate(offsets):
            cs, rs = max(0, k), max(0, -k)
            ln = min(m - cs, n - rs)
            if ln > 0:
                data[p, cs:cs + ln] = torch.diagonal(a, k)[:ln]
        return cls(data, offsets, (n, m))

    def todense(self) -> torch.Tensor:
        n, m = self.shape
        out = torch.zeros((n, m), dtype=torch.float64, device=self.data.device)
        for p, k in enumerate(self.offsets):
            cs, rs = max(0, k), max(0, -k)
            ln = min(m - cs, n - rs)
            if ln > 0:
                idx = torch.arange(ln, device=out.device)
                out[rs + idx, cs + idx] = self.data[p, cs:cs + ln]
        return out

    def _apply(self, x: torch.Tensor, axis: int, transpose: bool) -> torch.Tensor:
        _require_cuda(self.data, x)
        n, m = self.shape
        axis = axis % x.dim()
        m_in = n if transpose else m
        n_out = m if transpose else n
        if x.shape[axis] != m_in:
            raise ValueError(f"x.shape[{axis}] must be {m_in}")
        cplx = x.is_complex()
        x = x.to(torch.complex128 if cplx else torch.float64).contiguous()
        outer = 1
        for s in x.shape[:axis]:
            outer *= s
        inner = 1
        for s in x.shape[axis + 1:]:
            inner *= s
        out_shape = list(x.shape)
        out_shape[axis] = n_out
        y = torch.empty(out_shape, dtype=x.dtype, device=x.device)
        offs = _lib.int64_array(self.offsets)
        _lib.call("jfb_dia_matvec", self.data.data_ptr(), offs, len(self.offsets), n, m,
                  x.data_ptr(), y.data_ptr(), outer, inner, int(cplx), int(transpose),
                  _stream(x))
        return y

    def matvec(self, x: torch.Tensor, axis: int = 0) -> torch.Tensor:
        """``A`` applied along ``axis`` of ``x`` (diamatrix.py:227-283)."""
        return self._apply(x, axis, False)

    def rmatvec(self, x: torch.Tensor, axis: int = -1) -> torch.Tensor:
        """``x @ A`` contracting ``axis`` of ``x`` (diamatrix.py:285-348)."""
        return self._apply(x, axis, True)

    def __matmul__(self, x: torch.Tensor) -> torch.Tensor:
        return self.matvec(x, 0)

    def lu_factor(self, *, pivot: bool = False) -> LUFactors:
        """No-pivot banded LU, cached (diamatrix.py:394-504)."""
        if pivot:
            raise NotImplementedError("pivoted LU is not on the B200 path")
        if self._lu is None:
            n, m = self.shape
            if n != m:
                raise ValueError("lu_factor requires a square matrix")
            L, U, loffs, uoffs = _factor_batch(self.data.unsqueeze(0), self.offsets, n)
            self._lu = LUFactors(L[0], U[0], loffs, uoffs, n)
        return self._lu

    def solve(self, b: torch.Tensor, axis: int = 0) -> torch.Tensor:
        return self.lu_factor().solve(b, axis)


def _factor_batch(data: torch.Tensor, offsets: Sequence[int], n: int):
    """Batched no-pivot banded LU of DIA data (n_batch, n_diags, n) and the
    reference's pruning of all-zero diagonals (tpmatrix.py:1105-1149)."""
    p = max((-o for o in offsets if o < 0), default=0)
    q = max((o for o in offsets if o > 0), default=0)
    nb = data.shape[0]
    band = torch.zeros((nb, p + q + 1, n), dtype=torch.float64, device=data.device)
    for d, off in enumerate(offsets):
        band[:, p + off, :] = data[:, d, :]
    band = band.contiguous()
    _lib.call("jfb_banded_lu_factor", band.data_ptr(), nb, p, q, n, _stream(band))
    nz = (band != 0).any(dim=2).any(dim=0).cpu().tolist()
    l_offs = tuple(o for o in range(-p, 0) if nz[p + o])
    u_offs = tuple(o for o in range(0, q + 1) if nz[p + o] or o == 0)
    L = (band[:, [p + o for o in l_offs], :].contiguous() if l_offs
         else torch.zeros((nb, 0, n), dtype=torch.float64, device=data.device))
    U = band[:, [p + o for o in u_offs], :].contiguous()
    return L, U, l_offs, u_offs


class LUFactors:
    """Unit-lower ``L`` and upper ``U`` DIA factors (diamatrix.py:1855-1933)."""

    def __init__(self, L, U, L_offsets, U_offsets, n):
        self.L_data, self.U_data = L, U
        self.L_offsets, self.U_offsets = tuple(L_offsets), tuple(U_offsets)
        self.shape = (n, n)
        self.L = DiaMatrix(torch.cat([torch.ones((1, n), dtype=torch.float64, device=U.device), L])
                           if L.shape[0] else torch.ones((1, n), dtype=torch.float64,
                                                         device=U.device),
                           (0, *self.L_offsets) if L.shape[0] else (0,), (n, n))
        self.U = DiaMatrix(U, self.U_offsets, (n, n))

    def solve(self, b: torch.Tensor, axis: int = 0) -> torch.Tensor:
        """Forward then back substitution along ``axis``."""
        _require_cuda(b)
        n = self.shape[0]
        axis = axis % b.dim()
        bm = torch.movedim(b, axis, -1).contiguous()
        rest = bm.shape[:-1]
        k = 1
        for s in rest:
            k *= s
        cplx = bm.is_complex()
        bm = bm.to(torch.complex128 if cplx else torch.float64).reshape(k, n).contiguous()
        out = torch.empty_like(bm)
        lo, uo = _lib.int64_array(self.L_offsets), _lib.int64_array(self.U_offsets)
        L = self.L_data.contiguous()
        U = self.U_data.contiguous()
        # one factor shared by k right-hand sides: n_F = 1, n_rhs = k
        _lib.call("jfb_wavenumber_solve", L.data_ptr() if L.numel() else None, lo,
                  len(self.L_offsets), U.data_ptr(), uo, len(self.U_offsets), n, 1, 1, k,
                  bm.data_ptr(), out.data_ptr(), int(cplx), _stream(bm))
        return torch.movedim(out.reshape(*rest, n), -1, axis)


class TPMatrix:
    """``coefficient * mats[0] (x) mats[1] (x) ...`` (tpmatrix.py:40-200)."""

    def __init__(self, mats: Sequence[DiaMatrix], coefficient: float = 1.0):
        self.mats = list(mats)
        self.coefficient = float(coefficient)

    @property
    def dims(self) -> int:
        return len(self.mats)

    def __matmul__(self, u: torch.Tensor) -> torch.Tensor:
        r = u
        for i, mat in enumerate(self.mats):
            r = mat.matvec(r, axis=i)
        return r * self.coefficient


class TPMatrices:
    """Sum of ``TPMatrix`` terms (tpmatrix.py:300-428)."""

    def __init__(self, tpmats: Sequence[TPMatrix]):
        self.tpmats = list(tpmats)

    def __matmul__(self, u: torch.Tensor) -> torch.Tensor:
        out = None
        for tp in self.tpmats:
            r = tp @ u
            out = r if out is None else out + r
        return out

    def lu_factor(self) -> TPMatricesWavenumberSolver:
        return tpmats_wavenumber_factor(self)

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        return self.lu_factor().solve(rhs)


def tpmats_wavenumber_factor(A, *, pivot: bool = False, constraints=()) -> TPMatricesWavenumberSolver:
    """Per-wavenumber banded LU of a Fourier x polynomial system
    (tpmatrix.py:1900-2029).  The Fourier weights W[t, k] and the stacked
    polynomial DIA data are assembled as in the reference; the batched LU runs
    on the GPU."""
    if pivot or constraints:
        raise NotImplementedError("pivoted / constrained wavenumber solves are not on the B200 path")
    tpmats = list(A.tpmats) if isinstance(A, TPMatrices) else list(A)
    ndim = tpmats[0].dims

    def diagonal_axis(a):
        return all(set(tp.mats[a].offsets) == {0} for tp in tpmats)

    fourier = [a for a in range(ndim) if diagonal_axis(a)]
    poly = [a for a in range(ndim) if not diagonal_axis(a)]
    if len(poly) != 1:
        raise SolverNotApplicable(
            f"tpmats_wavenumber_factor requires exactly 1 polynomial axis; found {poly}"
        )
    pa = poly[0]
    shape = tuple(tpmats[0].mats[a].shape[0] for a in range(ndim))
    n_P = shape[pa]
    dev = tpmats[0].mats[pa].data.device
    W = []
    for tp in tpmats:
        w = torch.tensor([tp.coefficient], dtype=torch.float64, device=dev)
        for a in fourier:
            w = torch.outer(w, tp.mats[a].data[0].to(dev)).flatten()
        W.append(w)
    W = torch.stack(W)
    offs = sorted({int(o) for tp in tpmats for o in tp.mats[pa].offsets})
    P = torch.zeros((len(tpmats), len(offs), n_P), dtype=torch.float64, device=dev)
    for t, tp in enumerate(tpmats):
        mat = tp.mats[pa]
        for d, o in enumerate(offs):
            if o in mat.offsets:
                P[t, d] = mat.data[mat.offsets.index(o)]
    B = torch.einsum("tf,tdp->fdp", W, P).contiguous()
    return TPMatricesWavenumberSolver(pa, shape, B, tuple(offs))


class TPMatricesWavenumberSolver:
    """Per-Fourier-mode no-pivot banded solver (tpmatrix.py:1034-1677)."""

    def __init__(self, poly_axis: int, shape, B_data_batch: torch.Tensor,
                 poly_offsets: Sequence[int]):
        self.poly_axis = int(poly_axis)
        self.shape = tuple(int(s) for s in shape)
        n_P = self.shape[self.poly_axis]
        L, U, lo, uo = _factor_batch(B_data_batch, poly_offsets, n_P)
        self._L_data_local, self._U_data_local = L, U
        self.L_offsets, self.U_offsets = lo, uo
        self.wavenumber_backend = "b200"
        self._solve_args = (L, U)

    def _geom(self):
        pa = self.poly_axis
        outer = 1
        for s in self.shape[:pa]:
            outer *= s
        inner = 1
        for s in self.shape[pa + 1:]:
            inner *= s
        return outer, self.shape[pa], inner

    def _run(self, rhs: torch.Tensor, n_rhs: int, L, U) -> torch.Tensor:
        _require_cuda(rhs, L, U)
        outer, n_P, inner = self._geom()
        cplx = rhs.is_complex()
        r = rhs.to(torch.complex128 if cplx else torch.float64).contiguous()
        out = torch.empty_like(r)
        if not hasattr(self, "_offset_arrays"):
            self._offset_arrays = (_lib.int64_array(self.L_offsets),
                                   _lib.int64_array(self.U_offsets))
        lo, uo = self._offset_arrays
        L = L.contiguous()
        U = U.contiguous()
        _lib.call("jfb_wavenumber_solve", L.data_ptr() if L.numel() else None, lo,
                  len(self.L_offsets), U.data_ptr(), uo, len(self.U_offsets), n_P, outer,
                  inner, n_rhs, r.data_ptr(), out.data_ptr(), int(cplx), _stream(r))
        return out

    def solve(self, rhs: torch.Tensor) -> torch.Tensor:
        if tuple(rhs.shape) != self.shape:
            raise ValueError(f"rhs must have shape {self.shape}, received {tuple(rhs.shape)}")
        return self._run(rhs, 1, *self._solve_args)

    def solve_many(self, rhs: torch.Tensor) -> torch.Tensor:
        if rhs.dim() != len(self.shape) + 1 or tuple(rhs.shape[1:]) != self.shape:
            raise ValueError(
                f"multi-RHS input must have shape (n_rhs, {self.shape}), received {tuple(rhs.shape)}"
            )
        return self._run(rhs, rhs.shape[0], *self._solve_args)

    def runtime_args(self):
        return self._solve_args

    def solve_with_runtime_args(self, rhs, factor_args):
        if tuple(rhs.shape) != self.shape:
            raise ValueError(f"rhs must have shape {self.shape}")
        return self._run(rhs, 1, *factor_args)

    def solve_many_with_runtime_args(self, rhs, factor_args):
        if rhs.dim() != len(self.shape) + 1 or tuple(rhs.shape[1:]) != self.shape:
            raise ValueError(f"multi-RHS input must have shape (n_rhs, {self.shape})")
        return self._run(rhs, rhs.shape[0], *factor_args)
