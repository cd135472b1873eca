"""Tensor-product spaces (Chebyshev-family x Fourier [x Fourier]) and the
2-D Helmholtz solver, backed by ``libjfb200.so``.

``TensorProductSpace`` mirrors ``jaxfun.galerkin.TensorProductSpace``
(tensorproductspace.py:104-594) for the spaces of the hot path: ``backward``,
``forward``, ``scalar_product`` (padded or not) on full complex spectra in the
reference layout.  ``Helmholtz2D`` is the Shen-Galerkin solver of
``-lap u + alpha u = f`` (la/solvers.py:22-61 with the per-wavenumber banded
solve of tpmatrix.py:1550-1677): scalar products of f, one banded solve per
Fourier mode, backward transform.  All arithmetic runs on the GPU; there is no
CPU path.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .la import DiaMatrix, TPMatrices, TPMatrix, tpmats_wavenumber_factor

_BASES = {"C": _lib.JFB_BASIS_ORTHOGONAL, "D": _lib.JFB_BASIS_DIRICHLET,
          "B": _lib.JFB_BASIS_BIHARMONIC}


def _stream(dev) -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


class TensorProductSpace:
    """``TensorProduct(x_space, Fourier[, Fourier])``.

    basis: "C" (the orthogonal basis of the family), "D" (Dirichlet),
    "B" (biharmonic); family: "C" (Chebyshev) or "L" (Legendre: Gauss-Legendre
    nodes, Vandermonde contractions, orthogonal.py:121-145, 240-331);
    N = (x points, Fourier modes...); domain = ((x_lo, x_hi), (y0, y1)[, (z0, z1)]);
    padding_factor as in ``get_dealiased`` (the x entry is ignored).
    """

    def __init__(self, basis: str, N, domain, padding_factor=None, device="cuda",
                 family: str = "C"):
        self.N = tuple(int(n) for n in N)
        self.ndim = len(self.N)
        if self.ndim not in (2, 3):
            raise ValueError("2-D or 3-D spaces only")
        if basis not in _BASES:
            raise ValueError("basis must be 'C', 'D' or 'B'")
        self.basis = basis
        fam = str(family).upper()[:1]
        if fam not in ("C", "L"):
            raise ValueError("family must be 'C' (Chebyshev) or 'L' (Legendre)")
        self.family = fam
        self.domain = tuple(tuple(float(v) for v in d) for d in domain)
        pad = tuple(padding_factor) if padding_factor is not None else (1.0,) * self.ndim
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the transforms run on a CUDA device only")
        cfg = _lib.TPSConfig()
        cfg.ndim = self.ndim
        cfg.basis = _BASES[basis]
        cfg.family = _lib.JFB_FAMILY_LEGENDRE if fam == "L" else _lib.JFB_FAMILY_CHEBYSHEV
        for a in range(3):
            cfg.n[a] = self.N[a] if a < self.ndim else 1
        cfg.x_lo, cfg.x_hi = self.domain[0]
        for a in range(self.ndim - 1):
            cfg.l[a] = self.domain[a + 1][1] - self.domain[a + 1][0]
            cfg.pad[a] = float(pad[a + 1])
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.call("jfb_tps_create", ctypes.byref(cfg), ctypes.byref(h))
        self._h = h
        sizes = (ctypes.c_int32 * 4)()
        _lib.call("jfb_tps_get_sizes", h, sizes)
        self.num_dofs = (sizes[0],) + self.N[1:]
        self.padded_counts = (sizes[1], sizes[2]) + ((sizes[3],) if self.ndim == 3 else ())
        self.counts = self.N

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                _lib.load().jfb_tps_destroy(h)
            except Exception:
                pass
            self._h = None

    def _check(self, t: torch.Tensor, shape) -> torch.Tensor:
        if not t.is_cuda:
            raise ValueError("arrays must live on a CUDA device")
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {tuple(shape)}, received {tuple(t.shape)}")
        return t.to(torch.complex128).contiguous()

    def backward(self, c: torch.Tensor, padded: bool = False) -> torch.Tensor:
        c = self._check(c, self.num_dofs)
        shape = self.padded_counts if padded else self.counts
        out = torch.empty(shape, dtype=torch.complex128, device=self.device)
        _lib.call("jfb_tps_backward", self._h, c.data_ptr(), out.data_ptr(), int(padded),
                  _stream(self.device))
        return out

    def _fwd(self, u: torch.Tensor, padded: bool, kind: int) -> torch.Tensor:
        u = self._check(u, self.padded_counts if padded else self.counts)
        out = torch.empty(self.num_dofs, dtype=torch.complex128, device=self.device)
        _lib.call("jfb_tps_forward", self._h, u.data_ptr(), out.data_ptr(), int(padded), kind,
                  _stream(self.device))
        return out

    def forward(self, u: torch.Tensor, padded: bool = False) -> torch.Tensor:
        return self._fwd(u, padded, 0)

    def scalar_product(self, u: torch.Tensor, padded: bool = False) -> torch.Tensor:
        return self._fwd(u, padded, 1)

    def _orders(self, k) -> ctypes.Array:
        k = tuple(int(v) for v in k)
        if len(k) != self.ndim:
            raise ValueError(f"expected {self.ndim} derivative orders, received {len(k)}")
        if any(v < 0 for v in k):
            raise ValueError("derivative orders must be non-negative")
        return (ctypes.c_int32 * 3)(*(k + (0,) * (3 - len(k))))

    @property
    def orthogonal_shape(self):
        return (self.N[0],) + self.N[1:]

    def backward_primitive(self, c: torch.Tensor, k, padded: bool = False) -> torch.Tensor:
        """Mixed derivative of the field on the (padded) mesh
        (tensorproductspace.py:553-594)."""
        kk = self._orders(k)
        c = self._check(c, self.num_dofs)
        shape = self.padded_counts if padded else self.counts
        out = torch.empty(shape, dtype=torch.complex128, device=self.device)
        _lib.call("jfb_tps_backward_primitive", self._h, c.data_ptr(), out.data_ptr(), kk,
                  int(padded), _stream(self.device))
        return out

    def _coeff_map(self, name, c, shape_in, shape_out, *extra) -> torch.Tensor:
        c = self._check(c, shape_in)
        out = torch.empty(shape_out, dtype=torch.complex128, device=self.device)
        _lib.call(name, self._h, c.data_ptr(), out.data_ptr(), *extra, _stream(self.device))
        return out

    def to_orthogonal(self, c: torch.Tensor) -> torch.Tensor:
        """``c @ S`` along x (tensorproductspace.py:596-616)."""
        return self._coeff_map("jfb_tps_to_orthogonal", c, self.num_dofs, self.orthogonal_shape)

    def differentiate_orthogonal_coeffs(self, c: torch.Tensor, k) -> torch.Tensor:
        """tensorproductspace.py:638-682."""
        return self._coeff_map("jfb_tps_differentiate_orthogonal", c, self.orthogonal_shape,
                               self.orthogonal_shape, self._orders(k))

    def derivative_orthogonal_coeffs(self, c: torch.Tensor, k) -> torch.Tensor:
        """tensorproductspace.py:618-636."""
        return self.differentiate_orthogonal_coeffs(self.to_orthogonal(c), k)

    def project_from_orthogonal(self, c: torch.Tensor) -> torch.Tensor:
        """tensorproductspace.py:706-728."""
        return self._coeff_map("jfb_tps_project_from_orthogonal", c, self.orthogonal_shape,
                               self.num_dofs)

    def scalar_product_from_orthogonal(self, c: torch.Tensor) -> torch.Tensor:
        """tensorproductspace.py:730-754."""
        return self._coeff_map("jfb_tps_scalar_product_from_orthogonal", c,
                               self.orthogonal_shape, self.num_dofs)

    def galerkin(self, order: int) -> np.ndarray:
        """Dense (phi_i, phi_j^(order))_w along x (host array)."""
        nb = self.num_dofs[0]
        out = (ctypes.c_double * (nb * nb))()
        _lib.call("jfb_tps_galerkin", self._h, int(order), out)
        return np.frombuffer(out, dtype=np.float64).reshape(nb, nb).copy()

    def wavenumbers(self, axis: int) -> torch.Tensor:
        """Physical Fourier wavenumbers (FFT order) along a periodic axis."""
        n = self.N[axis]
        L = self.domain[axis][1] - self.domain[axis][0]
        k = torch.fft.fftfreq(n, d=1.0 / n, dtype=torch.float64)
        return (k * (2.0 * math.pi / L)).to(self.device)


class Helmholtz2D:
    """``-lap u + alpha u = f`` on Chebyshev-Dirichlet (x) x Fourier (y)
    (la/solvers.py:22-61): scalar products of f, one banded Galerkin solve
    per Fourier mode (``TPMatricesWavenumberSolver``), backward transform."""

    def __init__(self, N=(64, 64), domain=((-1.0, 1.0), (0.0, 2.0 * math.pi)),
                 alpha: float = 1.0, device="cuda"):
        self.TD = TensorProductSpace("D", N, domain, device=device)
        self.TC = TensorProductSpace("C", N, domain, device=device)
        self.device = self.TD.device
        G0, G2 = self.TD.galerkin(0), self.TD.galerkin(2)
        k = self.TD.wavenumbers(1)
        M = int(N[1])
        dev = self.device
        ident = DiaMatrix(torch.ones((1, M), dtype=torch.float64, device=dev), [0], (M, M))
        kk = DiaMatrix((k * k + alpha).reshape(1, M), [0], (M, M))

        def dia(a):  # every structurally nonzero diagonal, however small
            n = a.shape[0]
            offs = [k for k in range(-(n - 1), n) if np.any(np.diagonal(a, k) != 0.0)]
            return DiaMatrix.from_dense(torch.from_numpy(a).to(dev), offsets=offs)

        A = TPMatrices([TPMatrix([dia(-G2), ident]), TPMatrix([dia(G0), kk])])
        self.solver = tpmats_wavenumber_factor(A)
        # the Fourier mass 2 pi / df = L of the scalar product is not in A
        self._fourier_mass = domain[1][1] - domain[1][0]
        # one-launch path (jfb_helmholtz2d_solve) while the problem fits the
        # shared memory of one CTA cluster; the separate launches otherwise
        L, U = self.solver.runtime_args()
        self._L, self._U = L.contiguous(), U.contiguous()
        self._offs = (_lib.int64_array(self.solver.L_offsets),
                      _lib.int64_array(self.solver.U_offsets))
        props = torch.cuda.get_device_properties(self.device)
        optin = getattr(props, "shared_memory_per_block_optin", 0)
        n, m, nb = self.TD.N[0], self.TD.N[1], self.TD.num_dofs[0]
        kc, jr = -(-m // 8), -(-n // 8)  # columns / rows per CTA of the 8-CTA cluster
        qs = kc + (5 - kc % 4) % 4  # padded row of the solve vectors
        need = 16 * (2 * n * kc + n * qs + 2 * m * jr) + 8 * n * nb
        self.fused = need <= optin
        # explicit inverse of each mode's U (entry (r, c) at c nb + r): the
        # back substitution of the one-launch solve becomes a product
        self._Uinv = None
        if self.fused and nb <= 128:
            offs = torch.tensor(self.solver.U_offsets, device=self.device)
            Ud = self._U  # (modes, n_diag, nb): U[i, i + s] at [d, i + s]
            dense = torch.zeros((Ud.shape[0], nb, nb), dtype=torch.float64, device=self.device)
            cols = torch.arange(nb, device=self.device)
            for d in range(Ud.shape[1]):
                s_ = int(offs[d])
                c = cols[s_:]
                dense[:, c - s_, c] = Ud[:, d, s_:]
            eye = torch.eye(nb, dtype=torch.float64, device=self.device).expand_as(dense)
            inv = torch.linalg.solve_triangular(dense, eye, upper=True)
            self._Uinv = inv.transpose(1, 2).contiguous()

    def solve_coefficients(self, f_phys: torch.Tensor) -> torch.Tensor:
        """Dirichlet x Fourier coefficients of u from samples of f."""
        rhs = self.TD.scalar_product(f_phys) / self._fourier_mass
        return self.solver.solve(rhs)

    def __call__(self, f_hat: torch.Tensor) -> torch.Tensor:
        """f given by orthogonal Chebyshev x Fourier coefficients: backward,
        scalar products, per-mode solves, backward; returns u on the mesh.
        One launch (the whole problem in the shared memory of one 8-CTA
        cluster) when it fits, else the separate transforms and the
        wavenumber solve."""
        if not self.fused:
            return self.separate(f_hat)
        f = self.TC._check(f_hat, self.TC.num_dofs)
        u = torch.empty(self.TD.N, dtype=torch.complex128, device=self.device)
        lo, uo = self._offs
        _lib.call("jfb_helmholtz2d_solve", self.TC._h, self.TD._h,
                  self._L.data_ptr() if self._L.numel() else None, lo,
                  len(self.solver.L_offsets), self._U.data_ptr(), uo,
                  len(self.solver.U_offsets),
                  self._Uinv.data_ptr() if self._Uinv is not None else None,
                  self._fourier_mass, f.data_ptr(), u.data_ptr(), _stream(self.device))
        return u

    def separate(self, f_hat: torch.Tensor) -> torch.Tensor:
        """The same solve as separate launches: TC.backward, scalar products,
        jfb_wavenumber_solve, TD.backward."""
        f_phys = self.TC.backward(f_hat)
        return self.TD.backward(self.solve_coefficients(f_phys))

    def graphed(self, f_hat: torch.Tensor):
        """One solve captured in a CUDA graph: returns (graph, f_in, u_out);
        copy new forcing coefficients into f_in, replay the graph, read u_out
        (the launches of a solve replay without host work in between)."""
        f_in = f_hat.to(torch.complex128).clone().contiguous()
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(2):
                self(f_in)
        torch.cuda.current_stream(self.device).wait_stream(side)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            u_out = self(f_in)
        return g, f_in, u_out
