"""The CPU oracle against the reference's own recorded values (CPU only)."""

import json
import os

import numpy as np
import pytest

from oracle.kmm import PlaneCouetteMHDOracle, PlaneCouetteOracle

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "reference_goldens.json")))


def _solver(spec):
    s = spec["solver"]
    return PlaneCouetteOracle(
        N=tuple(s["N"]), family=s["family"], dt=s["dt"], Re=s["Re"],
        perturbation_amplitude=s["perturbation_amplitude"],
        time_integrator=s["time_integrator"], nonlinear_form=s["nonlinear_form"],
        coefficient_path=s["coefficient_path"], padding_factor=tuple(s["padding_factor"]),
    )


def test_one_step_legendre_golden():
    """tests/couette/test_pcf_fluctuations_jax.py:218-238 of the reference."""
    spec = GOLD["one_step_legendre_9x8x8"]
    o = _solver(spec)
    d = o.diagnostics(o.step(o.initial_state()))
    for key, value in spec["diagnostics"].items():
        atol = 1e-12 if key != "divL2" else 5e-15
        assert np.isclose(d[key], value, rtol=spec["rtol"], atol=atol), key


@pytest.mark.slow
def test_benchmark_325_steps_golden():
    """benchmark-results/hydro-sbdf3-rotational-65x64x64-r2.json of the
    reference: 13 blocks x 25 SBDF3 rotational steps (about 4 minutes)."""
    spec = GOLD["benchmark_hydro_sbdf3_rotational_65x64x64"]
    o = _solver(spec)
    st = o.solve(o.initial_state(), spec["steps"])
    d = o.diagnostics(st)
    for key in ("Epert", "Etot", "wall_shear_top", "wall_shear_bot", "u_top", "u_bot"):
        assert np.isclose(d[key], spec["diagnostics"][key], rtol=1e-10, atol=1e-14), key
    leaves = (list(st.u) + [st.g] + list(st.nonlinear_old) + list(st.nonlinear_older)
              + list(st.solution_old) + list(st.solution_older))
    count = sum(a.size for a in leaves) + 3
    l2 = np.sqrt(sum(float(np.sum(np.abs(a) ** 2)) for a in leaves) + 4.0 + 1.0
                 + spec["solver"]["dt"] ** 2)
    cs = spec["state_checksum"]
    assert count == cs["element_count"]
    assert np.isclose(l2, cs["l2_norm"], rtol=1e-10)


@pytest.mark.slow
def test_mhd_benchmark_325_steps_golden():
    """benchmark-results/mhd-sbdf3-rotational-65x64x64-r1.json of the
    reference: the coupled flow + vector-potential step, 325 SBDF3 rotational
    steps (about 10 minutes)."""
    spec = GOLD["benchmark_mhd_sbdf3_rotational_65x64x64"]
    s = spec["solver"]
    o = PlaneCouetteMHDOracle(N=tuple(s["N"]), Re=s["Re"], Rm=s["Rm"], dt=s["dt"],
                              perturbation_amplitude=s["perturbation_amplitude"],
                              magnetic_amplitude=s["magnetic_amplitude"])
    d = o.diagnostics(o.solve(o.initial_state(), spec["steps"]))
    for key in ("Emag", "Epert", "Etot", "wall_shear_top", "wall_shear_bot", "u_top", "u_bot"):
        assert np.isclose(d[key], spec["diagnostics"][key], rtol=1e-10, atol=1e-14), key
    assert d["divB_L2"] < 1e-15 and d["divL2"] < 1e-15


def test_oracle_matches_committed_fixture():
    """Regression of the oracle against tests/golden/pcf_17x16x16.npz."""
    fx = np.load(os.path.join(HERE, "golden", "pcf_17x16x16.npz"))
    o = PlaneCouetteOracle(N=(17, 16, 16), Re=600.0, dt=0.01, perturbation_amplitude=0.05)
    st = o.initial_state()
    for n in range(11):
        if n in (0, 3, 10):
            for i in range(3):
                np.testing.assert_allclose(st.u[i], fx[f"s{n}_u{i}"], rtol=0, atol=1e-14)
            np.testing.assert_allclose(st.g, fx[f"s{n}_g"], rtol=0, atol=1e-14)
        st = o.step(st)
