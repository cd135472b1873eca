"""ctypes binding of ``libjfb200.so`` (the C ABI declared in include/jfb200.h).

The shared library is built in-tree by ``jaxfun_b200.build.build()``.  There is
no fallback: importing a function from this module when the library is
missing raises ``ImportError`` with the build command to run.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_int32, c_int64, c_void_p

_HERE = os.path.dirname(os.path.abspath(__file__))
# JFB200_LIB may name another in-tree build of the same library (the
# phase-stamp build, libjfb200_stamps.so, for profiling).
LIB_PATH = os.environ.get("JFB200_LIB") or os.path.join(_HERE, "libjfb200.so")

JFB_OK = 0
JFB_ERR_ARG = 1
JFB_ERR_CUDA = 2
JFB_ERR_SINGULAR = 3
JFB_ERR_NONFINITE = 4
JFB_ERR_STATE = 5
JFB_ERR_DEVICE = 6

JFB_FAMILY_CHEBYSHEV = 0
JFB_PRECISION_FP64 = 0
JFB_PRECISION_MIXED = 1
JFB_NONLINEAR_ROTATIONAL = 0
JFB_NONLINEAR_GRADIENT = 1
JFB_INTEGRATOR_SBDF3 = 0
JFB_INTEGRATOR_IMEXRK3 = 1
JFB_INTEGRATOR_IMEXRK222 = 2
JFB_INTEGRATOR_CNAB2 = 3
JFB_BASIS_ORTHOGONAL = 0
JFB_BASIS_DIRICHLET = 1
JFB_BASIS_BIHARMONIC = 2
JFB_FAMILY_LEGENDRE = 1


class KMMConfig(ctypes.Structure):
    """``jfb_kmm_config`` (include/jfb200.h)."""

    _fields_ = [
        ("nx", c_int32),
        ("ny", c_int32),
        ("nz", c_int32),
        ("family", c_int32),
        ("x_lo", c_double),
        ("x_hi", c_double),
        ("ly", c_double),
        ("lz", c_double),
        ("pad_y", c_double),
        ("pad_z", c_double),
        ("nu", c_double),
        ("dt", c_double),
        ("u_wall", c_double),
        ("precision", c_int32),
        ("nonlinear_form", c_int32),
        ("time_integrator", c_int32),
    ]


class KMMStateC(ctypes.Structure):
    """``jfb_kmm_state``: device pointers of a KMMState in the reference layout."""

    _fields_ = [
        ("u0", c_void_p),
        ("u1", c_void_p),
        ("u2", c_void_p),
        ("g", c_void_p),
        ("nonlinear_old", c_void_p * 4),
        ("nonlinear_older", c_void_p * 4),
        ("solution_old", c_void_p * 4),
        ("solution_older", c_void_p * 4),
        ("history_steps", c_double),
    ]


class MHDStateC(ctypes.Structure):
    """``jfb_mhd_state``: device pointers of an MHDState in the reference layout."""

    _fields_ = [
        ("flow", KMMStateC),
        ("A", c_void_p * 3),
        ("nonlinear_A_old", c_void_p * 3),
        ("nonlinear_A_older", c_void_p * 3),
        ("A_old", c_void_p * 3),
        ("A_older", c_void_p * 3),
    ]


class MHDParams(ctypes.Structure):
    """``jfb_mhd_params``."""

    _fields_ = [
        ("eta", c_double),
        ("omega", c_double),
        ("b0", c_double * 3),
    ]


class TPSConfig(ctypes.Structure):
    """``jfb_tps_config``."""

    _fields_ = [
        ("ndim", c_int32),
        ("basis", c_int32),
        ("n", c_int32 * 3),
        ("x_lo", c_double),
        ("x_hi", c_double),
        ("l", c_double * 2),
        ("pad", c_double * 2),
        ("family", c_int32),
    ]


class KMMVariant(ctypes.Structure):
    """``jfb_kmm_variant``: kernel choices of a flow plan."""

    _fields_ = [
        ("pencil", c_int32),
        ("transforms", c_int32),
        ("tc_velocity", c_int32),
        ("pdl", c_int32),
        ("replicas", c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: int(getattr(self, name)) for name, _ in self._fields_}


class KMMInfo(ctypes.Structure):
    _fields_ = [
        ("n_pencils", c_int64),
        ("device_bytes", c_int64),
        ("launches_per_step", c_int64),
        ("algorithmic_bytes", c_int64),
        ("my", c_int32),
        ("mz", c_int32),
    ]


# name -> (restype, argtypes); every symbol declared in include/jfb200.h
SIGNATURES = {
    "jfb_version": (c_int, []),
    "jfb_last_error": (ctypes.c_char_p, []),
    "jfb_dia_matvec": (
        c_int,
        [c_void_p, POINTER(c_int64), c_int64, c_int64, c_int64, c_void_p, c_void_p,
         c_int64, c_int64, c_int, c_int, c_void_p],
    ),
    "jfb_banded_lu_factor": (
        c_int, [c_void_p, c_int64, c_int64, c_int64, c_int64, c_void_p]
    ),
    "jfb_banded_lu_factor_noalloc": (
        c_int, [c_void_p, c_int64, c_int64, c_int64, c_int64, POINTER(c_int32), c_void_p]
    ),
    "jfb_wavenumber_solve": (
        c_int,
        [c_void_p, POINTER(c_int64), c_int64, c_void_p, POINTER(c_int64), c_int64,
         c_int64, c_int64, c_int64, c_int64, c_void_p, c_void_p, c_int, c_void_p],
    ),
    "jfb_kmm_create": (c_int, [POINTER(KMMConfig), POINTER(c_void_p)]),
    "jfb_kmm_destroy": (c_int, [c_void_p]),
    "jfb_kmm_get_info": (c_int, [c_void_p, POINTER(KMMInfo)]),
    "jfb_kmm_set_state": (c_int, [c_void_p, POINTER(KMMStateC), c_void_p]),
    "jfb_kmm_get_state": (c_int, [c_void_p, POINTER(KMMStateC), c_void_p]),
    "jfb_kmm_advance": (c_int, [c_void_p, c_int64, c_void_p]),
    "jfb_kmm_convection": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "jfb_kmm_state_from_physical": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "jfb_kmm_diagnostics": (c_int, [c_void_p, c_void_p, c_void_p]),
    "jfb_kmm_check": (c_int, [c_void_p, POINTER(c_int32), c_void_p]),
    "jfb_kmm_get_variant": (c_int, [c_void_p, POINTER(KMMVariant), POINTER(KMMVariant)]),
    "jfb_kmm_set_variant": (c_int, [c_void_p, POINTER(KMMVariant)]),
    "jfb_kmm_autotune": (
        c_int, [c_void_p, c_int64, POINTER(KMMVariant), POINTER(c_double), c_void_p]
    ),
    "jfb_kmm_timed_steps": (
        c_int,
        [c_void_p, c_int64, c_void_p, c_int64, POINTER(c_double), POINTER(c_double), c_void_p],
    ),
    "jfb_kmm_gain_gradient": (
        c_int,
        [c_void_p, POINTER(KMMStateC), c_int64, c_int64, POINTER(c_double),
         POINTER(KMMStateC), c_void_p],
    ),
    "jfb_kmm_energy_gradient": (
        c_int, [c_void_p, POINTER(KMMStateC), POINTER(KMMStateC), c_void_p]
    ),
    "jfb_mhd_create": (c_int, [POINTER(KMMConfig), POINTER(MHDParams), POINTER(c_void_p)]),
    "jfb_tps_create": (c_int, [POINTER(TPSConfig), POINTER(c_void_p)]),
    "jfb_tps_destroy": (c_int, [c_void_p]),
    "jfb_tps_get_sizes": (c_int, [c_void_p, POINTER(c_int32)]),
    "jfb_tps_backward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p]),
    "jfb_tps_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p]),
    "jfb_tps_galerkin": (c_int, [c_void_p, c_int, POINTER(c_double)]),
    "jfb_tps_backward_primitive": (
        c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_int32), c_int, c_void_p]
    ),
    "jfb_tps_to_orthogonal": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "jfb_tps_differentiate_orthogonal": (
        c_int, [c_void_p, c_void_p, c_void_p, POINTER(c_int32), c_void_p]
    ),
    "jfb_tps_project_from_orthogonal": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "jfb_tps_scalar_product_from_orthogonal": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "jfb_helmholtz2d_solve": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int64,
                                       c_void_p, c_void_p, c_int64, c_void_p, c_double,
                                       c_void_p, c_void_p, c_void_p]),
    "jfb_ensemble_create": (c_int, [POINTER(c_void_p), c_int32, POINTER(c_void_p)]),
    "jfb_ensemble_advance": (c_int, [c_void_p, c_int64, c_void_p]),
    "jfb_ensemble_info": (c_int, [c_void_p, POINTER(c_int32), POINTER(c_int64)]),
    "jfb_ensemble_destroy": (c_int, [c_void_p]),
    "jfb_mhd_set_state": (c_int, [c_void_p, POINTER(MHDStateC), c_void_p]),
    "jfb_mhd_get_state": (c_int, [c_void_p, POINTER(MHDStateC), c_void_p]),
    "jfb_mhd_potential_from_physical": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "jfb_mhd_convection": (
        c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]
    ),
    "jfb_mhd_diagnostics": (c_int, [c_void_p, c_void_p, c_void_p]),
}

_lib = None


def load() -> ctypes.CDLL:
    """Load (once) and return the shared library; raise if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with "
            "`python -c 'import jaxfun_b200.build as b; b.build()'`"
        )
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class JFBError(RuntimeError):
    """A non-zero status returned by the C ABI."""

    def __init__(self, status: int, msg: str):
        super().__init__(f"jfb status {status}: {msg}")
        self.status = status


class NonFiniteStateError(JFBError, FloatingPointError):
    """JFB_ERR_NONFINITE: the state holds NaN or infinite values.  A
    ``FloatingPointError``, as the reference's runner raises for a non-finite
    solver state (production/oracles.py:3257-3261)."""


def check(status: int) -> None:
    if status != JFB_OK:
        msg = load().jfb_last_error()
        text = msg.decode() if msg else ""
        if status == JFB_ERR_NONFINITE:
            raise NonFiniteStateError(status, text)
        raise JFBError(status, text)


def call(name: str, *args) -> None:
    """Call a C-ABI function and raise ``JFBError`` on a non-zero status."""
    check(getattr(load(), name)(*args))


def int64_array(values) -> ctypes.Array:
    vals = [int(v) for v in values]
    return (c_int64 * max(1, len(vals)))(*vals)
