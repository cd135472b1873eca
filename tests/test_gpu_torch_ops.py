"""The torch.library operators of jaxfun_b200.torch_ops on the GPU: results
equal the ctypes-level calls, and their autograd formulas equal the
transposed product (DIA matvec) and the hand-written adjoint (gain)."""

import math

import numpy as np
import pytest
import torch

from jaxfun_b200 import minimal_seed as ms
from jaxfun_b200 import torch_ops
from jaxfun_b200.kmm import PlaneCouetteFluctuation
from jaxfun_b200.la import DiaMatrix
from jaxfun_b200.tps import TensorProductSpace

pytestmark = pytest.mark.gpu
ops = torch.ops.jaxfun_b200


def test_dia_matvec_op_and_its_gradient(cuda):
    g = torch.Generator().manual_seed(3)
    n, m, offs = 21, 19, [-2, 0, 1, 4]
    data = torch.randn((len(offs), m), generator=g, dtype=torch.float64).to(cuda)
    x = torch.randn((5, m, 3), generator=g, dtype=torch.complex128).to(cuda)
    A = DiaMatrix(data, offs, (n, m))
    y = ops.dia_matvec(data, offs, n, m, x, 1, False)
    assert torch.equal(y, A.matvec(x, axis=1))
    xr = x.real.contiguous().requires_grad_(True)
    w = torch.randn((5, n, 3), generator=g, dtype=torch.float64).to(cuda)
    (ops.dia_matvec(data, offs, n, m, xr, 1, False) * w).sum().backward()
    dense = A.todense()
    ref = torch.einsum("in,bik->bnk", dense, w)
    assert torch.allclose(xr.grad, ref, rtol=1e-13, atol=1e-13)
    torch.library.opcheck(ops.dia_matvec.default, (data, offs, n, m, x, 1, False),
                          test_utils=("test_schema", "test_faketensor"))


def test_wavenumber_solve_op_matches_dense_solves(cuda):
    g = torch.Generator().manual_seed(4)
    nF, nP = 7, 12
    Lo, Uo = [-2], [0, 2]
    L = 0.1 * torch.randn((nF, 1, nP), generator=g, dtype=torch.float64)
    U = torch.randn((nF, 2, nP), generator=g, dtype=torch.float64)
    U[:, 0] += 5.0
    rhs = torch.randn((nF, nP), generator=g, dtype=torch.complex128)
    x = ops.wavenumber_solve(L.to(cuda), Lo, U.to(cuda), Uo, rhs.to(cuda)).cpu()
    for f in range(nF):  # column-aligned DIA: data[d, j] = A[j - off, j]
        Lm, Um = torch.eye(nP, dtype=torch.float64), torch.zeros((nP, nP), dtype=torch.float64)
        for j in range(nP):
            if j + 2 < nP:
                Lm[j + 2, j] = L[f, 0, j]
            Um[j, j] = U[f, 0, j]
            if j >= 2:
                Um[j - 2, j] = U[f, 1, j]
        ref = torch.linalg.solve((Lm @ Um).to(torch.complex128), rhs[f])
        assert torch.allclose(x[f], ref, rtol=1e-12, atol=1e-12)


def test_tps_ops_match_space_methods(cuda):
    T = TensorProductSpace("D", (17, 16, 12), ((-1.0, 1.0), (0.0, 2 * math.pi), (0.0, 2 * math.pi)),
                           padding_factor=(1.0, 1.5, 1.5), device=cuda)
    h = torch_ops.register_space(T)
    rng = np.random.default_rng(1)
    c = torch.from_numpy(rng.standard_normal(T.num_dofs) + 1j * rng.standard_normal(T.num_dofs))
    c = c.to(cuda)
    try:
        u = ops.tps_backward(h, c, True)
        assert torch.equal(u, T.backward(c, padded=True))
        assert torch.equal(ops.tps_forward(h, u, True, 0), T.forward(u, padded=True))
        assert torch.equal(ops.tps_forward(h, u, True, 1), T.scalar_product(u, padded=True))
    finally:
        torch_ops.unregister(h)


def test_kmm_gain_op_backward_is_the_adjoint(cuda):
    s = PlaneCouetteFluctuation(N=(17, 16, 16), Re=400.0, dt=0.01, perturbation_amplitude=0.1,
                                device=cuda, time_integrator="SBDF3", nonlinear_form="rotational")
    x0 = s.initial_state()
    h = torch_ops.register_solver(s)
    try:
        leaves = [t.clone().requires_grad_(True) for t in (*x0.u, x0.g)]
        gain = ops.kmm_gain(h, 6, 2, *leaves)
        ref_gain, grad = ms.gain_and_gradient(s, ms._primary(x0), 6, checkpoint=2)
        assert abs(gain.item() - ref_gain) <= 1e-14 * abs(ref_gain)
        gain.backward()
        for t, gj in zip(leaves, (*grad.u, grad.g), strict=True):
            assert torch.allclose(t.grad, gj.conj(), rtol=0, atol=1e-13 * gj.abs().max().item())
    finally:
        torch_ops.unregister(h)
