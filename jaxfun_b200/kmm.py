"""KMM / plane-Couette solver objects backed by the sm_100a step.

Mirrors the reference's public API for the hot path:
``examples/channelflow_kmm.py`` (``KMM``, ``KMMState``: ``step``, ``solve``,
``convection``, ``zero_state``) and ``examples/pcf_fluctuations_jax.py``
(``PlaneCouetteFluctuationJax``).  Arrays are torch tensors on a CUDA device in
the reference layout (wall-normal axis first, full complex Fourier axes).
All arithmetic runs in ``libjfb200.so``; there is no CPU path.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, replace

import numpy as np
import torch

from . import _lib
from .cadence import Cadence, run_with_cadence

_STEPPERS = {"IMEXRK222", "IMEXRK3", "CNAB2", "SBDF3"}
_GPU_STEPPERS = {"SBDF3": _lib.JFB_INTEGRATOR_SBDF3, "IMEXRK3": _lib.JFB_INTEGRATOR_IMEXRK3,
                 "IMEXRK222": _lib.JFB_INTEGRATOR_IMEXRK222,
                 "CNAB2": _lib.JFB_INTEGRATOR_CNAB2}


@dataclass(frozen=True)
class KMMState:
    """Coefficient-space state with SBDF3 history (channelflow_kmm.py:50-101)."""

    u: tuple
    g: torch.Tensor
    nonlinear_old: tuple | None = None
    nonlinear_older: tuple | None = None
    solution_old: tuple | None = None
    solution_older: tuple | None = None
    history_steps: float = 0.0
    have_old: float = 0.0  # CNAB2: nonlinear_old holds N(u^(n-1))
    previous_dt: float = 0.0


def _ptr(t: torch.Tensor | None) -> int | None:
    if t is None:
        return None
    if not t.is_cuda:
        raise ValueError("KMM state tensors must live on a CUDA device")
    if not t.is_contiguous():
        raise ValueError("KMM state tensors must be contiguous")
    return t.data_ptr()


class KMM:
    """Velocity-vorticity KMM channel solver (channelflow_kmm.py:104-230).

    Same constructor defaults as the reference: gradient nonlinear form,
    ``time_integrator=None`` meaning IMEXRK222, the "transform" coefficient
    path.  Supported on the GPU path: Chebyshev or Legendre family,
    wall-normal axis unpadded, the gradient form ``u . grad u`` or the
    rotational form ``-(u x omega)``, each in FP64 or mixed precision; time
    integrators SBDF3 (IMEXRK3 startup), IMEXRK3, IMEXRK222 (the one-step
    integrators keep no history: the state's history fields pass through
    unchanged, as in the reference's ``KMM.step``) and CNAB2 with the
    plan's fixed ``dt`` (``nonlinear_old``, ``have_old`` and ``previous_dt``
    carry its history, as in the reference's ``_cnab2_flow_update``).  The coefficient path
    ("optimized" or "transform") only changes round-off in the reference
    (tests/couette/test_pcf_fluctuations_jax.py:16-52), so both names select
    the same coefficient-space kernels.
    """

    def __init__(
        self,
        N=(17, 16, 16),
        domain=((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi)),
        nu: float = 1.0 / 600.0,
        dt: float = 0.01,
        family: str = "C",
        padding_factor=(1.0, 1.5, 1.5),
        dpdy: float = 0.0,
        time_integrator: str | None = None,
        nonlinear_form: str = "gradient",
        coefficient_path: str = "transform",
        solve_batching: str = "batched",
        precision: str = "fp64",
        device: str | torch.device = "cuda",
        _u_wall: float = 0.0,
    ) -> None:
        self.N = tuple(int(n) for n in N)
        self.domain = tuple(tuple(float(v) for v in d) for d in domain)
        self.nu = float(nu)
        self.dt = float(dt)
        self.padding_factor = tuple(float(p) for p in padding_factor)
        self.nonlinear_form = str(nonlinear_form).lower()
        if self.nonlinear_form not in {"gradient", "rotational"}:
            raise ValueError("nonlinear_form must be 'gradient' or 'rotational'")
        self.coefficient_path = str(coefficient_path).lower()
        if self.coefficient_path not in {"optimized", "transform"}:
            raise ValueError("coefficient_path must be 'optimized' or 'transform'")
        if str(solve_batching).lower() not in {"batched", "separate"}:
            raise ValueError("solve_batching must be 'batched' or 'separate'")
        if time_integrator is not None and time_integrator not in _STEPPERS:
            raise ValueError(
                "time_integrator must be one of "
                "{'IMEXRK222', 'IMEXRK3', 'CNAB2', 'SBDF3'}"
            )
        # channelflow_kmm.py:149-193: no integrator named -> IMEXRK222
        if time_integrator is None:
            time_integrator = "IMEXRK222"
        fam = str(family).upper()[:1]
        if fam not in ("C", "L"):
            raise ValueError("family must be 'C' (Chebyshev) or 'L' (Legendre)")
        unsupported = []
        if time_integrator not in _GPU_STEPPERS:
            unsupported.append(f"time_integrator={time_integrator!r}")
        if self.padding_factor[0] != 1.0:
            unsupported.append("wall-normal padding")
        if float(dpdy) != 0.0:
            unsupported.append("dpdy != 0")
        if unsupported:
            raise NotImplementedError(
                "the B200 step supports SBDF3, IMEXRK3, IMEXRK222 or CNAB2 / unpadded x "
                "only; requested " + ", ".join(unsupported)
            )
        self.time_integrator = time_integrator
        self.family = fam
        self.precision = precision
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError("the B200 step runs on a CUDA device only")
        self.dpdy = 0.0
        Nx, Ny, Nz = self.N
        self.shape_B = (Nx - 4, Ny, Nz)
        self.shape_D = (Nx - 2, Ny, Nz)
        cfg = _lib.KMMConfig()
        cfg.nx, cfg.ny, cfg.nz = Nx, Ny, Nz
        cfg.family = _lib.JFB_FAMILY_LEGENDRE if fam == "L" else _lib.JFB_FAMILY_CHEBYSHEV
        cfg.x_lo, cfg.x_hi = self.domain[0]
        cfg.ly = self.domain[1][1] - self.domain[1][0]
        cfg.lz = self.domain[2][1] - self.domain[2][0]
        cfg.pad_y, cfg.pad_z = self.padding_factor[1], self.padding_factor[2]
        cfg.nu = self.nu
        cfg.dt = self.dt
        cfg.u_wall = float(_u_wall)
        cfg.precision = {
            "fp64": _lib.JFB_PRECISION_FP64,
            "mixed": _lib.JFB_PRECISION_MIXED,
        }[precision]
        cfg.nonlinear_form = (_lib.JFB_NONLINEAR_GRADIENT if self.nonlinear_form == "gradient"
                              else _lib.JFB_NONLINEAR_ROTATIONAL)
        cfg.time_integrator = _GPU_STEPPERS[self.time_integrator]
        self._cfg = cfg
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            self._create_plan(cfg, handle)
        self._plan = handle
        self._current = None  # the state object the plan currently holds

    def _create_plan(self, cfg: _lib.KMMConfig, handle: ctypes.c_void_p) -> None:
        _lib.call("jfb_kmm_create", ctypes.byref(cfg), ctypes.byref(handle))

    # -- plumbing -------------------------------------------------------------
    def __del__(self):
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.value:
            try:
                _lib.load().jfb_kmm_destroy(plan)
            except Exception:
                pass
            self._plan = None

    def _stream(self) -> ctypes.c_void_p:
        return ctypes.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def info(self) -> _lib.KMMInfo:
        info = _lib.KMMInfo()
        _lib.call("jfb_kmm_get_info", self._plan, ctypes.byref(info))
        return info

    def _c_state(self, st: KMMState) -> _lib.KMMStateC:
        c = _lib.KMMStateC()
        c.u0, c.u1, c.u2 = (_ptr(t) for t in st.u)
        c.g = _ptr(st.g)
        for name in ("nonlinear_old", "nonlinear_older", "solution_old", "solution_older"):
            lv = getattr(st, name)
            arr = getattr(c, name)
            for k in range(4):
                arr[k] = _ptr(lv[k]) if lv is not None else None
        c.history_steps = (float(bool(st.have_old)) if self.time_integrator == "CNAB2"
                           else float(st.history_steps))
        return c

    def _empty_state(self) -> KMMState:
        dev = self.device
        cd = torch.complex128

        def lv():
            return (
                torch.empty(self.shape_B, dtype=cd, device=dev),
                torch.empty(self.shape_D, dtype=cd, device=dev),
                torch.empty(self.shape_D[0], dtype=torch.float64, device=dev),
                torch.empty(self.shape_D[0], dtype=torch.float64, device=dev),
            )

        return KMMState(
            u=(
                torch.empty(self.shape_B, dtype=cd, device=dev),
                torch.empty(self.shape_D, dtype=cd, device=dev),
                torch.empty(self.shape_D, dtype=cd, device=dev),
            ),
            g=torch.empty(self.shape_D, dtype=cd, device=dev),
            nonlinear_old=lv(),
            nonlinear_older=lv(),
            solution_old=lv(),
            solution_older=lv(),
        )

    def _load(self, state: KMMState) -> None:
        if state is self._current:
            return
        state = self._ensure_history(state)
        c = self._c_state(state)
        _lib.call("jfb_kmm_set_state", self._plan, ctypes.byref(c), self._stream())
        self._current = state

    def _fetch(self, history_steps: float) -> KMMState:
        out = self._empty_state()
        out = replace(out, history_steps=float(history_steps))
        c = self._c_state(out)
        _lib.call("jfb_kmm_get_state", self._plan, ctypes.byref(c), self._stream())
        self._current = out
        return out

    def _ensure_history(self, state: KMMState) -> KMMState:
        """Zero history levels for a fresh state (channelflow_kmm.py:609-654)."""
        if state.solution_old is not None and state.nonlinear_old is not None:
            return state
        if self.time_integrator == "CNAB2" and state.nonlinear_old is not None:
            # CNAB2 keeps one nonlinear level; the plan's other levels are unused
            z = (
                torch.zeros_like(state.u[0]),
                torch.zeros_like(state.g),
                torch.zeros(self.shape_D[0], dtype=torch.float64, device=self.device),
                torch.zeros(self.shape_D[0], dtype=torch.float64, device=self.device),
            )
            return replace(state, nonlinear_older=z, solution_old=z, solution_older=z)
        z = (
            torch.zeros_like(state.u[0]),
            torch.zeros_like(state.g),
            torch.zeros(self.shape_D[0], dtype=torch.float64, device=self.device),
            torch.zeros(self.shape_D[0], dtype=torch.float64, device=self.device),
        )
        return replace(
            state,
            nonlinear_old=z,
            nonlinear_older=z,
            solution_old=z,
            solution_older=z,
            history_steps=0.0,
            have_old=0.0,
            previous_dt=0.0,
        )

    # -- reference API ----------------------------------------------------------
    def zero_state(self) -> KMMState:
        dev, cd = self.device, torch.complex128
        st = KMMState(
            u=(
                torch.zeros(self.shape_B, dtype=cd, device=dev),
                torch.zeros(self.shape_D, dtype=cd, device=dev),
                torch.zeros(self.shape_D, dtype=cd, device=dev),
            ),
            g=torch.zeros(self.shape_D, dtype=cd, device=dev),
        )
        return self._ensure_history(st)

    def step(self, state: KMMState, dt=None, factor_args=None) -> KMMState:
        """One step of the plan's integrator (SBDF3: IMEXRK3 startup while
        history_steps < 2).  The factors belong to the plan's fixed time
        step, so ``dt`` must be None or equal to it."""
        if dt is not None and float(dt) != self.dt:
            raise NotImplementedError("the B200 step runs the plan's fixed dt")
        return self.solve(state, 1)

    def solve(self, state: KMMState, steps: int) -> KMMState:
        """Advance ``steps`` steps (channelflow_kmm.py:1231-1247).

        Raises ``FloatingPointError`` (``_lib.NonFiniteStateError``) when a
        solved coefficient became NaN or infinite, as the reference's runner
        does for a non-finite state (production/oracles.py:3257-3261)."""
        steps = int(steps)
        if (self.time_integrator == "CNAB2" and state.have_old
                and float(state.previous_dt) not in (0.0, self.dt)):
            raise NotImplementedError(
                "CNAB2 history from a different step size (variable_ab2_extrapolate "
                "ratio != 1); the B200 plan runs a fixed dt")
        self._load(state)
        loaded = self._current
        hist = float(loaded.history_steps)
        _lib.call("jfb_kmm_advance", self._plan, steps, self._stream())
        if self.time_integrator == "SBDF3":
            out = self._fetch(min(2.0, hist + steps))
        elif self.time_integrator == "CNAB2":
            was = float(bool(loaded.have_old))
            out = self._fetch(0.0)
            if steps > 0:
                out = replace(out, have_old=1.0, previous_dt=self.dt,
                              nonlinear_older=None, solution_old=None, solution_older=None)
            else:
                out = replace(out, have_old=was, previous_dt=loaded.previous_dt,
                              nonlinear_older=None, solution_old=None, solution_older=None)
            self._current = out
        else:  # one-step integrators: the history fields pass through
            out = replace(self._fetch(hist), nonlinear_old=loaded.nonlinear_old,
                          nonlinear_older=loaded.nonlinear_older,
                          solution_old=loaded.solution_old,
                          solution_older=loaded.solution_older)
            self._current = out
        self.check()
        return out

    def solve_with_cadence(self, state, steps: int, cadence: Cadence, *, block_size: int = 1,
                           on_diagnostics=None, on_snapshot=None, on_checkpoint=None,
                           should_stop=None, t0: float = 0.0, tstep0: int = 0):
        """``solve`` in blocks with host callbacks at the cadence boundaries
        (channelflow_kmm.py:1264-1289; contract in ``jaxfun_b200.cadence``);
        the diagnostics passed to ``on_diagnostics`` are ``self.diagnostics``
        of the state at the boundary."""
        return run_with_cadence(
            self.solve, state, steps=steps, dt=self.dt, cadence=cadence,
            block_size=block_size, diagnostics=self.diagnostics,
            on_diagnostics=on_diagnostics, on_snapshot=on_snapshot,
            on_checkpoint=on_checkpoint, should_stop=should_stop, t0=t0, tstep0=tstep0,
        )

    def check(self) -> None:
        """Read and clear the plan's device status word (synchronises the
        stream); raise if a step saw a non-finite value or a timed-out wait."""
        _lib.call("jfb_kmm_check", self._plan, None, self._stream())

    # -- kernel variants -------------------------------------------------------
    def variant(self) -> dict:
        """The plan's kernel choices (``jfb_kmm_variant``) and the largest
        value each accepts."""
        cur, avail = _lib.KMMVariant(), _lib.KMMVariant()
        _lib.call("jfb_kmm_get_variant", self._plan, ctypes.byref(cur), ctypes.byref(avail))
        return {"current": cur.as_dict(), "available": avail.as_dict()}

    def set_variant(self, **fields) -> None:
        """Select kernel choices by field name (see ``jfb_kmm_variant``)."""
        v = _lib.KMMVariant(**self.variant()["current"])
        for k, val in fields.items():
            if not hasattr(v, k):
                raise ValueError(f"unknown variant field {k!r}")
            setattr(v, k, int(val))
        _lib.call("jfb_kmm_set_variant", self._plan, ctypes.byref(v))

    def autotune(self, state: KMMState | None = None, steps: int = 20,
                 cache: bool = True) -> dict:
        """Time every kernel variant this plan accepts on copies of ``state``
        (default: the loaded state), select the fastest and return
        ``{"variant": ..., "ms_per_step": ...}``.  With ``cache`` the choice
        is remembered per (device, grid, precision) in the file named by
        JFB200_AUTOTUNE_CACHE (default ~/.cache/jaxfun_b200/autotune.json)
        and reused without timing."""
        from . import autotune as at

        key = at.cache_key(self)
        if cache:
            hit = at.lookup(key)
            if hit is not None:
                try:
                    self.set_variant(**hit["variant"])
                    return dict(hit, cached=True)
                except _lib.JFBError:
                    pass
        if state is not None:
            self._load(state)
        if self._current is None:
            raise ValueError("autotune needs a state: pass one or load one first")
        best, ms = _lib.KMMVariant(), ctypes.c_double()
        _lib.call("jfb_kmm_autotune", self._plan, int(steps), ctypes.byref(best),
                  ctypes.byref(ms), self._stream())
        out = {"variant": best.as_dict(), "ms_per_step": ms.value, "cached": False}
        if cache:
            at.store(key, out)
        return out

    def advance_resident(self, steps: int) -> None:
        """Advance the device-resident state without materialising it."""
        _lib.call("jfb_kmm_advance", self._plan, int(steps), self._stream())
        self._current = None

    # -- meshes and physical-space entry points -------------------------------
    def mesh(self):
        """Quadrature mesh (x on the Gauss-Chebyshev or Gauss-Legendre nodes,
        y/z uniform), broadcast like ``TensorProductSpace.mesh``
        (tensorproductspace.py:207-232; Legendre.py:136-147 takes numpy's
        ``leggauss`` nodes)."""
        Nx, Ny, Nz = self.N
        (a, b), (y0, y1), (z0, z1) = self.domain
        if self.family == "L":
            X = torch.from_numpy(np.polynomial.legendre.leggauss(Nx)[0])
        else:
            X = torch.cos(
                math.pi + (2 * torch.arange(Nx, dtype=torch.float64) + 1) * math.pi / (2 * Nx)
            )
        x = a + (X + 1.0) * (b - a) / 2.0
        y = y0 + torch.arange(Ny, dtype=torch.float64) * (y1 - y0) / Ny
        z = z0 + torch.arange(Nz, dtype=torch.float64) * (z1 - z0) / Nz
        dev = self.device
        return (
            x.reshape(Nx, 1, 1).to(dev),
            y.reshape(1, Ny, 1).to(dev),
            z.reshape(1, 1, Nz).to(dev),
        )

    def state_from_physical(self, u_phys) -> KMMState:
        """``KMM.state_from_physical`` (channelflow_kmm.py:677-683): real
        velocity samples (Nx, Ny, Nz) on the quadrature mesh -> coefficient
        state with a zero history."""
        shape = self.N
        fields = []
        for v in u_phys:
            t = torch.as_tensor(v, device=self.device)
            if t.is_complex():
                t = t.real
            t = torch.broadcast_to(t.to(torch.float64), shape).contiguous()
            fields.append(t)
        _lib.call(
            "jfb_kmm_state_from_physical", self._plan, fields[0].data_ptr(),
            fields[1].data_ptr(), fields[2].data_ptr(), self._stream(),
        )
        return self._fetch(0.0)

    def diagnostics_tensor(self, state: KMMState) -> torch.Tensor:
        """Device tensor (8,) of the scalar diagnostics of ``state``."""
        self._load(state)
        out = torch.empty(8, dtype=torch.float64, device=self.device)
        _lib.call("jfb_kmm_diagnostics", self._plan, out.data_ptr(), self._stream())
        return out

    DIAGNOSTIC_NAMES = (
        "Epert", "Etot", "divL2", "u_top", "u_bot",
        "wall_shear_top", "wall_shear_bot", "mean_shear",
    )

    def diagnostics(self, state: KMMState) -> dict[str, float]:
        """pcf_fluctuations_jax.py:131-161 (with U_wall = 0 for the plain KMM)."""
        vals = self.diagnostics_tensor(state).cpu().tolist()
        return dict(zip(self.DIAGNOSTIC_NAMES, vals, strict=True))

    def perturbation_energy(self, state: KMMState) -> float:
        return self.diagnostics(state)["Epert"]

    def divergence_l2(self, state: KMMState) -> float:
        return self.diagnostics(state)["divL2"]

    def convection(self, state: KMMState):
        """Dealiased rotational convection in TD coefficients (channelflow_kmm.py:772-782)."""
        self._load(state)
        H = tuple(
            torch.empty(self.shape_D, dtype=torch.complex128, device=self.device)
            for _ in range(3)
        )
        _lib.call(
            "jfb_kmm_convection", self._plan, H[0].data_ptr(), H[1].data_ptr(),
            H[2].data_ptr(), self._stream(),
        )
        return H


class PlaneCouetteFluctuation(KMM):
    """Fluctuations about ``U_b = U_wall x`` (pcf_fluctuations_jax.py:29-75)."""

    def __init__(
        self,
        N=(17, 16, 16),
        domain=((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi)),
        Re: float = 600.0,
        U_wall: float = 1.0,
        dt: float = 0.01,
        family: str = "C",
        padding_factor=(1.0, 1.5, 1.5),
        perturbation_amplitude: float = 0.05,
        timestepper=None,
        time_integrator: str | None = None,
        nonlinear_form: str = "gradient",
        coefficient_path: str = "transform",
        solve_batching: str = "batched",
        precision: str = "fp64",
        device="cuda",
    ) -> None:
        self.Re = float(Re)
        self.U_wall = float(U_wall)
        self.perturbation_amplitude = float(perturbation_amplitude)
        super().__init__(
            N=N,
            domain=domain,
            nu=self.U_wall / self.Re,
            dt=dt,
            family=family,
            padding_factor=padding_factor,
            time_integrator=time_integrator,
            nonlinear_form=nonlinear_form,
            coefficient_path=coefficient_path,
            solve_batching=solve_batching,
            precision=precision,
            device=device,
            _u_wall=self.U_wall,
        )
        self.dUb_dx = self.U_wall

    def initial_state(self) -> KMMState:
        """Deterministic analytic perturbation (pcf_fluctuations_jax.py:77-97)."""
        x, y, z = self.mesh()
        amp = self.perturbation_amplitude
        wall = 1.0 - x**2
        Ly = self.domain[1][1] - self.domain[1][0]
        Lz = self.domain[2][1] - self.domain[2][0]
        tp = 2.0 * math.pi
        u0 = amp * wall * torch.sin(tp * y / Ly) * torch.cos(tp * z / Lz)
        u1 = amp * wall * torch.cos(tp * y / Ly) * torch.sin(tp * z / Lz)
        u2 = amp * wall * torch.sin(2 * tp * y / Ly) * torch.cos(2 * tp * z / Lz)
        return self.state_from_physical((u0, u1, u2))


# reference name
PlaneCouetteFluctuationJax = PlaneCouetteFluctuation
