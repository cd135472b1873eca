"""CPU FP64 oracle for the plane-Couette pseudo-spectral Galerkin step.

TEST INFRASTRUCTURE ONLY.  This package is a NumPy/SciPy restatement of the
reference algorithm (fnauman/jaxfun: the Chebyshev/Legendre/Fourier bases,
the Shen composite bases, the DIA banded no-pivot LU, the per-wavenumber
Kronecker solver and the KMM velocity-vorticity time step with its SBDF3,
IMEXRK3 and IMEXRK222 integrators).  It exists so that ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` can check
the CUDA implementation in ``jaxfun_b200`` against an independent computation.
The product package never imports it.

Parity pin: the reference cannot be executed here (JAX is not installed), so
the restatement is pinned against the reference's own recorded golden values:

* ``tests/couette/test_pcf_fluctuations_jax.py:218-238`` — one IMEXRK222 step
  of the Legendre (9, 8, 8) gradient/transform solver, scalar diagnostics at
  ``rtol 1e-10``;
* ``benchmark-results/hydro-sbdf3-rotational-65x64x64-r2.json`` —
  ``timing.final_diagnostics`` after 325 SBDF3 rotational steps of the
  Chebyshev 65x64x64 solver (Re=400, dt=1e-3, amplitude 0.02).

See ``tests/test_oracle_golden.py``.
"""

from .kmm import (  # noqa: F401
    Chebyshev1D,
    Composite1D,
    Fourier1D,
    KMMOracle,
    KMMState,
    Legendre1D,
    PlaneCouetteOracle,
    TensorSpace,
    WavenumberSolver,
)
