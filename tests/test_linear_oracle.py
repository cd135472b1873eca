"""The linear-stability oracle against the reference's recorded outputs and
unit tests (no GPU), and the host side of ``jaxfun_b200.linear``.

Goldens: ``tests/golden/reference_linear_goldens.json`` (expected-output
blocks of couette/couette_linear_benchmarks.md).  Unit cases:
tests/la/test_eig.py and tests/la/test_linear_analysis.py.
"""

import json
import math
from pathlib import Path

import numpy as np
import pytest

from jaxfun_b200.linear import PlaneCouetteLinear, legendre_kmm_matrices, parse_times
from oracle import linear as ol

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_linear_goldens.json").read_text())


@pytest.fixture(scope="module")
def re1000_nx96():
    return ol.PlaneCouetteLinearOracle.couette(nx=96, Re=1000.0)


def test_oracle_leading_growth_rates(re1000_nx96):
    for ky, kz, want in GOLD["leading_growth_re1000_nx96"]["cases"]:
        got = re1000_nx96.growth_rate(ky, kz)
        assert abs(got - want) <= 5e-7 * abs(want), (ky, kz, got, want)  # 7 printed digits


def test_oracle_streamwise_roll(re1000_nx96):
    nu = 1.0 / 1000.0
    for kz, want in GOLD["streamwise_roll_re1000_nx96"]["cases"]:
        w, _ = re1000_nx96.eigs(0.0, kz, n_return=4)
        assert abs(w[0].real - want) <= 5e-9 * abs(want)
        assert abs(w[0].real + nu * (kz * kz + (math.pi / 2) ** 2)) <= 1e-9 * abs(want)


def test_oracle_transient_growth_re1000():
    g = GOLD["transient_growth_re1000_nx80"]
    pcf = ol.PlaneCouetteLinearOracle.couette(nx=g["nx"], Re=g["Re"])
    row = pcf.nonmodal_growth(g["ky"], g["kz"], [139.0])[0]
    assert row["gain"] == pytest.approx(g["at_139"]["gain"], rel=1e-8)
    rows = pcf.nonmodal_growth(g["ky"], g["kz"], np.linspace(*g["best_scan"]["times"]))
    best = max(rows, key=lambda r: r["gain"])
    assert best["t"] == g["best_scan"]["t"]
    assert best["gain"] == pytest.approx(g["best_scan"]["gain"], rel=1e-8)


def test_oracle_optimal_growth_scaling_re500():
    g = GOLD["optimal_growth_scaling_nx80"]
    Re, gmax, topt = g["rows"][0]
    pcf = ol.PlaneCouetteLinearOracle.couette(nx=g["nx"], Re=Re)
    rows = pcf.nonmodal_growth(g["ky"], g["kz"], np.linspace(0.12 * Re, 0.40 * Re, 40))
    best = max(rows, key=lambda r: r["gain"])
    assert abs(best["gain"] - gmax) <= 0.006 and abs(best["t"] - topt) <= 0.06


def test_oracle_hydro_gain_and_its_metric_truncation():
    """The recorded G(50) at ky = kz = 1 comes from a modal basis with three
    nearly dependent directions dropped (metric_rtol 1e-10); kept, the gain
    is larger (the full propagator's value, which the product reports)."""
    g = GOLD["hydro_gain_re500_nx48"]
    pcf = ol.PlaneCouetteLinearOracle.couette(nx=g["nx"], Re=g["Re"])
    assert pcf.nonmodal_growth(g["ky"], g["kz"], [g["t"]])[0]["gain"] == pytest.approx(
        g["gain"], rel=1e-7)
    L, M = pcf.assemble(g["ky"], g["kz"])
    w, V = ol.finite_eigensystem(L, M)
    full = ol.transient_growth_from_eigs(w, V, pcf.energy_matrix(), [g["t"]], metric_rtol=1e-16)
    assert full[0]["gain"] > 1.04 * g["gain"]


# -- the reference's unit tests of la/eig.py, on the oracle --------------------

def test_oracle_parse_times_and_singular_mass():
    assert np.allclose(ol.parse_times("0, 1;2"), [0.0, 1.0, 2.0])
    for bad in ("", [0.0, -1.0]):
        with pytest.raises(ValueError):
            ol.parse_times(bad)
    w = ol.generalized_eig(np.diag([2.0, 3.0]), np.diag([1.0, 0.0]))
    assert w.shape == (1,) and np.allclose(w, [2.0])


def test_oracle_physical_eigensystem_filters_null_modes():
    L = np.diag([1.0e5, 0.5, -0.25]).astype(complex)
    values, vectors = ol.physical_eigensystem(L, np.eye(3, dtype=complex),
                                              np.diag([0.0, 2.0, 1.0]).astype(complex), n_return=2)
    assert values == pytest.approx([0.5, -0.25]) and vectors.shape == (3, 2)


# -- host side of the product module (no device compute) ---------------------

def test_parse_times_matches_the_oracle():
    for v in ("3;1, 2", [0.0, 0.5], np.array([4.0])):
        assert np.array_equal(parse_times(v), ol.parse_times(v))
    for bad in ("", " , ", [1.0, -2.0]):
        with pytest.raises(ValueError):
            parse_times(bad)


def test_legendre_kmm_basis_matrices():
    m = legendre_kmm_matrices(24)
    assert m["A0"].shape == (20, 20) and m["B0"].shape == (22, 22) and m["C"].shape == (22, 20)
    for k in ("A0", "A1", "A2", "X0", "B0", "B1", "XB"):
        assert np.abs(m[k] - m[k].T).max() <= 1e-14 * np.abs(m[k]).max(), k
    for k in ("A0", "A1", "A2", "B0", "B1"):
        assert np.linalg.eigvalsh(m[k]).min() > 0, k
    # the lowest biharmonic function phi_0 = L_0 - 10/7 L_2 + 3/7 L_4 vanishes with its
    # slope at the walls; its A0 and A1 entries against a trapezoid sum
    x = np.linspace(-1, 1, 2001)
    phi0 = np.polynomial.legendre.Legendre([1.0, 0.0, -10.0 / 7.0, 0.0, 3.0 / 7.0])
    assert abs(phi0(1.0)) < 1e-14 and abs(phi0.deriv()(1.0)) < 1e-14
    assert m["A0"][0, 0] == pytest.approx(np.trapezoid(phi0(x) ** 2, x), rel=1e-5)
    assert m["A1"][0, 0] == pytest.approx(np.trapezoid(phi0.deriv()(x) ** 2, x), rel=1e-5)
    with pytest.raises(ValueError):
        legendre_kmm_matrices(5)


def test_operator_options_rejected_before_device_work():
    with pytest.raises(ValueError, match="magnetic_bc"):
        PlaneCouetteLinear(nx=16, magnetic_bc="vacuum", device="meta")
    hydro = PlaneCouetteLinear.couette(nx=16, Re=100.0, device="meta")
    with pytest.raises(ValueError, match="mhd=True"):
        hydro.energy_matrix("magnetic", ky=1.0, kz=1.0)
    with pytest.raises(ValueError, match="kind"):
        hydro.energy_matrix("enstrophy", ky=1.0, kz=1.0)
    mhd = PlaneCouetteLinear.shearpy(nx=16, device="meta")
    assert mhd.mhd and mhd.n == 8 * 16 and mhd.Uprime == -1.0
    with pytest.raises(ValueError, match="nx"):
        PlaneCouetteLinear.couette(nx=3, mhd=True, device="meta")


def test_product_collocation_matrices_match_the_oracle():
    """The MHD operator's Chebyshev-Lobatto points, derivative matrix and
    Clenshaw-Curtis weights (host arrays) against the oracle's."""
    from jaxfun_b200.linear import cheb_lobatto

    for n in (5, 8, 33):
        for a, b in zip(cheb_lobatto(n), ol.cheb_lobatto(n), strict=True):
            assert np.allclose(a, b, rtol=1e-13, atol=1e-12)
    x, D, D2, w = cheb_lobatto(17)
    assert abs(w.sum() - 2.0) < 1e-14
    assert np.allclose(D @ x ** 3, 3 * x ** 2, atol=1e-11)


def test_oracle_mhd_energy_norms():
    g = GOLD["mhd_energy_norms_re500_nx48"]
    T = [g["t"]]
    mhd = ol.PlaneCouetteLinearOracle.couette(nx=g["nx"], Re=g["Re"], Rm=g["Rm"], mhd=True)
    for kind in ("kinetic", "magnetic", "total"):
        got = mhd.nonmodal_growth(g["ky"], g["kz"], T, energy=kind)[0]["gain"]
        assert got == pytest.approx(g["B0_zero"][kind], rel=1e-7), kind
    for bz, want in g["bz_sweep_total"][1:]:
        m = ol.PlaneCouetteLinearOracle.couette(nx=g["nx"], Re=g["Re"], Rm=g["Rm"], mhd=True, bz=bz)
        assert m.nonmodal_growth(g["ky"], g["kz"], T)[0]["gain"] == pytest.approx(want, rel=5e-7)


def test_oracle_shearpy_mri_growth_rate():
    g = GOLD["shearpy_mri_lead_eigenvalue"]
    kz = math.sqrt(15.0 / 16.0) * g["omega"] / g["bz"]
    for nx, want in g["lead"][:2]:
        lin = ol.PlaneCouetteLinearOracle.shearpy(nx=nx, Re=g["Re"], Rm=g["Rm"],
                                                  shear_rate=g["shear_rate"], omega=g["omega"],
                                                  by=g["by"], bz=g["bz"])
        w, _ = lin.eigs(0.0, kz, n_return=3)
        assert abs(w[0] - want) <= 1e-10


def test_oracle_magnetic_wall_conditions_are_stable():
    """Every wall condition gives a finite, decaying leading mode for a
    weak imposed field at moderate Re (smoke check of the wall rows)."""
    for bc in ol.PlaneCouetteLinearOracle.BCS:
        m = ol.PlaneCouetteLinearOracle.couette(nx=24, Re=200.0, Rm=200.0, mhd=True, bz=0.05,
                                                magnetic_bc=bc)
        r = m.growth_rate(1.0, 1.0)
        assert math.isfinite(r) and r < 0.0, bc


def test_growth_order_and_finite_filter_match_the_oracle():
    """Ordering by descending real part, ties by descending imaginary part
    (la/eig.py:12-19), and the finite-cap filter, on index arrays only."""
    import torch

    from jaxfun_b200.linear import _growth_sort, _keep_finite

    rng = np.random.default_rng(7)
    re = rng.integers(-3, 3, 40).astype(float)          # many equal real parts
    im = rng.integers(-2, 3, 40).astype(float)
    w = re + 1j * im
    got = _growth_sort(torch.as_tensor(w)).numpy()
    want = ol.growth_order(w)
    assert np.array_equal(w[got], w[want])
    v = torch.tensor([1.0 + 0j, complex(math.inf, 0), 5e6 + 0j, -2.0 + 1j, complex(0, math.nan)])
    kept, _ = _keep_finite(v, None, 1e6)
    assert kept.tolist() == [1.0 + 0j, -2.0 + 1j]
