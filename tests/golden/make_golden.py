"""Regenerate the golden fixtures of tests/golden/.

reference_goldens.json holds scalar values recorded BY THE REFERENCE
(fnauman/jaxfun) in its own test suite and benchmark artefacts, copied with
their source locations; they pin the oracle.  pcf_17x16x16.npz holds oracle
states (the CPU restatement, itself pinned by those scalars) used to check the
CUDA path.  Run from the repository root:  python tests/golden/make_golden.py
"""

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.kmm import PlaneCouetteOracle  # noqa: E402

REFERENCE = {
    "one_step_legendre_9x8x8": {
        "source": "tests/couette/test_pcf_fluctuations_jax.py:218-238",
        "solver": {"N": [9, 8, 8], "family": "L", "dt": 1.0e-3,
                   "perturbation_amplitude": 0.05, "Re": 600.0,
                   "time_integrator": "IMEXRK222", "nonlinear_form": "gradient",
                   "coefficient_path": "transform", "padding_factor": [1.0, 1.5, 1.5]},
        "steps": 1,
        "diagnostics": {"Epert": 0.21836099019180652, "Etot": 52.85625108205688,
                        "divL2": 7.183953559387109e-17, "u_top": 1.0, "u_bot": -1.0,
                        "mean_shear": 1.0},
        "rtol": 1e-10,
    },
    "benchmark_hydro_sbdf3_rotational_65x64x64": {
        "source": "benchmark-results/hydro-sbdf3-rotational-65x64x64-r2.json "
                  "(timing.final_diagnostics, timing.state_checksum)",
        "solver": {"N": [65, 64, 64], "family": "C", "dt": 1.0e-3,
                   "perturbation_amplitude": 0.02, "Re": 400.0,
                   "time_integrator": "SBDF3", "nonlinear_form": "rotational",
                   "coefficient_path": "optimized", "padding_factor": [1.0, 1.5, 1.5]},
        "steps": 325,
        "diagnostics": {"Epert": 0.03186035144205132, "Etot": 52.66915370319814,
                        "divL2": 7.724318055264452e-17, "mean_shear": 1.0,
                        "u_bot": -1.0, "u_top": 1.0,
                        "wall_shear_bot": 1.0000166621380333,
                        "wall_shear_top": 1.0000166621380333},
        "state_checksum": {"element_count": 3056123, "l2_norm": 5.062610681087452,
                           "real_sum": -7.830872524041756},
    },
    "benchmark_mhd_sbdf3_rotational_65x64x64": {
        "source": "benchmark-results/mhd-sbdf3-rotational-65x64x64-r1.json "
                  "(timing.final_diagnostics; solver built by "
                  "production/benchmark_pcf_refactor.py: PlaneCouetteMHDJax, "
                  "velocity amplitude 0.02, magnetic amplitude 0.005)",
        "solver": {"N": [65, 64, 64], "family": "C", "dt": 1.0e-3,
                   "perturbation_amplitude": 0.02, "magnetic_amplitude": 0.005,
                   "Re": 400.0, "Rm": 400.0,
                   "time_integrator": "SBDF3", "nonlinear_form": "rotational",
                   "coefficient_path": "optimized", "padding_factor": [1.0, 1.5, 1.5]},
        "steps": 325,
        "diagnostics": {"Emag": 0.0006539729631867507, "Epert": 0.03186034627195483,
                        "Etot": 52.669153697981685, "divB_L2": 3.2078792579026027e-18,
                        "divL2": 7.275547313434249e-17, "mean_shear": 1.0,
                        "u_bot": -1.0, "u_top": 1.0,
                        "wall_shear_bot": 1.0000166621379911,
                        "wall_shear_top": 1.0000166621379911},
    },
}


def main():
    with open(os.path.join(HERE, "reference_goldens.json"), "w") as f:
        json.dump(REFERENCE, f, indent=1)
    o = PlaneCouetteOracle(N=(17, 16, 16), Re=600.0, dt=0.01, perturbation_amplitude=0.05)
    st = o.initial_state()
    out = {}
    diags = []
    for n in range(11):
        if n in (0, 3, 10):
            for i, a in enumerate(st.u):
                out[f"s{n}_u{i}"] = a
            out[f"s{n}_g"] = st.g
        d = o.diagnostics(st)
        diags.append([d[k] for k in sorted(d)])
        st = o.step(st)
    out["diag_names"] = np.array(sorted(o.diagnostics(st)))
    out["diagnostics"] = np.array(diags)
    np.savez_compressed(os.path.join(HERE, "pcf_17x16x16.npz"), **out)


if __name__ == "__main__":
    main()
