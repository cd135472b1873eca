"""Plane-Couette MHD backed by the sm_100a coupled step.

Mirrors ``examples/pcf_mhd_jax.py`` (``MHDState``, ``PlaneCouetteMHDJax``):
the magnetic field is carried by its vector potential A in the Dirichlet
basis (conducting walls), B = curl A and J = curl B are formed in coefficient
space, the Lorentz force -J x B enters the momentum nonlinear term and the EMF
(u + U_b e_y) x B drives A.  Arrays are torch tensors on a CUDA device in the
reference layout.  All arithmetic runs in ``libjfb200.so``; there is no CPU
path.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, replace

import torch

from . import _lib
from .kmm import KMMState, PlaneCouetteFluctuation, _ptr


@dataclass(frozen=True)
class MHDState:
    """Coefficient-space MHD state with SBDF3 history (pcf_mhd_jax.py:34-66)."""

    flow: KMMState
    A: tuple
    nonlinear_A_old: tuple | None = None
    nonlinear_A_older: tuple | None = None
    A_old: tuple | None = None
    A_older: tuple | None = None


class PlaneCouetteMHD(PlaneCouetteFluctuation):
    """Plane Couette MHD with A as the evolved magnetic unknown
    (pcf_mhd_jax.py:69-790).  GPU path: SBDF3 with IMEXRK3 startup,
    rotational nonlinear form, Chebyshev family, FP64."""

    DIAGNOSTIC_NAMES = PlaneCouetteFluctuation.DIAGNOSTIC_NAMES + ("divB_L2", "Emag")

    def __init__(
        self,
        N=(17, 16, 16),
        domain=((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi)),
        Re: float = 400.0,
        Rm: float | None = None,
        U_wall: float = 1.0,
        dt: float = 0.01,
        family: str = "C",
        padding_factor=(1.0, 1.5, 1.5),
        perturbation_amplitude: float = 0.1,
        magnetic_amplitude: float = 0.05,
        time_integrator: str | None = "SBDF3",
        nonlinear_form: str = "rotational",
        coefficient_path: str = "transform",
        solve_batching: str = "batched",
        device="cuda",
    ) -> None:
        self.Rm = float(Re if Rm is None else Rm)
        self.eta = float(U_wall) / self.Rm
        self.magnetic_amplitude = float(magnetic_amplitude)
        super().__init__(
            N=N,
            domain=domain,
            Re=Re,
            U_wall=U_wall,
            dt=dt,
            family=family,
            padding_factor=padding_factor,
            perturbation_amplitude=perturbation_amplitude,
            time_integrator=time_integrator,
            nonlinear_form=nonlinear_form,
            coefficient_path=coefficient_path,
            solve_batching=solve_batching,
            precision="fp64",
            device=device,
        )

    def _create_plan(self, cfg: _lib.KMMConfig, handle: ctypes.c_void_p) -> None:
        _lib.call("jfb_mhd_create", ctypes.byref(cfg), self.Rm, ctypes.byref(handle))

    # -- plumbing -------------------------------------------------------------
    def _c_mhd_state(self, st: MHDState) -> _lib.MHDStateC:
        c = _lib.MHDStateC()
        c.flow = self._c_state(st.flow)
        for name in ("A", "nonlinear_A_old", "nonlinear_A_older", "A_old", "A_older"):
            lv = getattr(st, name)
            arr = getattr(c, name)
            for k in range(3):
                arr[k] = _ptr(lv[k]) if lv is not None else None
        return c

    def _zero_A(self):
        return tuple(
            torch.zeros(self.shape_D, dtype=torch.complex128, device=self.device)
            for _ in range(3)
        )

    def _empty_A(self):
        return tuple(
            torch.empty(self.shape_D, dtype=torch.complex128, device=self.device)
            for _ in range(3)
        )

    def _ensure_mhd_history(self, state: MHDState) -> MHDState:
        """pcf_mhd_jax.py:217-248: flow and A histories form one SBDF3
        timeline; if either is incomplete, both restart."""
        flow = state.flow
        complete = (
            state.nonlinear_A_old is not None
            and state.nonlinear_A_older is not None
            and state.A_old is not None
            and state.A_older is not None
            and flow.solution_old is not None
            and flow.nonlinear_old is not None
        )
        if complete:
            return state
        flow = self._ensure_history(replace(flow, solution_old=None))
        z = self._zero_A()
        return replace(state, flow=flow, nonlinear_A_old=z, nonlinear_A_older=z, A_old=z,
                       A_older=z)

    def _load(self, state) -> None:
        if state is self._current:
            return
        if isinstance(state, KMMState):
            raise TypeError("PlaneCouetteMHD operates on MHDState")
        state = self._ensure_mhd_history(state)
        c = self._c_mhd_state(state)
        _lib.call("jfb_mhd_set_state", self._plan, ctypes.byref(c), self._stream())
        self._current = state

    def _fetch_mhd(self, history_steps: float) -> MHDState:
        flow = replace(self._empty_state(), history_steps=float(history_steps))
        out = MHDState(flow=flow, A=self._empty_A(), nonlinear_A_old=self._empty_A(),
                       nonlinear_A_older=self._empty_A(), A_old=self._empty_A(),
                       A_older=self._empty_A())
        c = self._c_mhd_state(out)
        _lib.call("jfb_mhd_get_state", self._plan, ctypes.byref(c), self._stream())
        self._current = out
        return out

    # -- reference API ----------------------------------------------------------
    def _A_state_from_physical(self, a_phys) -> tuple:
        """pcf_mhd_jax.py:210-215: TD.forward (Nyquist masked) of real samples."""
        fields = []
        for v in a_phys:
            t = torch.as_tensor(v, device=self.device)
            if t.is_complex():
                t = t.real
            fields.append(torch.broadcast_to(t.to(torch.float64), self.N).contiguous())
        A = self._empty_A()
        _lib.call(
            "jfb_mhd_potential_from_physical", self._plan, *(f.data_ptr() for f in fields),
            *(a.data_ptr() for a in A), self._stream(),
        )
        return A

    def initial_state(self) -> MHDState:
        """pcf_mhd_jax.py:253-267: the flow seed plus
        A_x = amp (1 - x^2) sin(ky y) sin(kz z) / kz."""
        flow = super().initial_state()
        x, y, z = self.mesh()
        amp = self.magnetic_amplitude
        zero = torch.zeros(self.N, dtype=torch.float64, device=self.device)
        ax = zero
        if amp != 0.0:
            Ly = self.domain[1][1] - self.domain[1][0]
            Lz = self.domain[2][1] - self.domain[2][0]
            ky, kz = 2.0 * math.pi / Ly, 2.0 * math.pi / Lz
            ax = amp * (1.0 - x**2) * (1.0 / kz) * torch.sin(ky * y) * torch.sin(kz * z)
        A = self._A_state_from_physical((ax, zero, zero))
        return self._ensure_mhd_history(MHDState(flow=flow, A=A))

    def solve(self, state: MHDState, steps: int) -> MHDState:
        """Advance ``steps`` coupled steps (IMEXRK3 startup, then SBDF3)."""
        steps = int(steps)
        self._load(state)
        hist = float(self._current.flow.history_steps)
        _lib.call("jfb_kmm_advance", self._plan, steps, self._stream())
        return self._fetch_mhd(min(2.0, hist + steps))

    def step(self, state: MHDState, dt=None, factor_args=None) -> MHDState:
        return self.solve(state, 1)

    def diagnostics_tensor(self, state: MHDState) -> torch.Tensor:
        """Device tensor (10,): the flow diagnostics, divB_L2, Emag."""
        self._load(state)
        out = torch.empty(10, dtype=torch.float64, device=self.device)
        _lib.call("jfb_mhd_diagnostics", self._plan, out.data_ptr(), self._stream())
        return out

    def diagnostics(self, state: MHDState) -> dict[str, float]:
        """pcf_mhd_jax.py:776-790."""
        vals = self.diagnostics_tensor(state).cpu().tolist()
        return dict(zip(self.DIAGNOSTIC_NAMES, vals, strict=True))

    def magnetic_divergence_l2(self, state: MHDState) -> float:
        return self.diagnostics(state)["divB_L2"]

    def convection(self, state: MHDState):
        """_mhd_convection (pcf_mhd_jax.py:339-357): (H, HA) in TD coefficients."""
        self._load(state)
        out = tuple(
            torch.empty(self.shape_D, dtype=torch.complex128, device=self.device)
            for _ in range(6)
        )
        _lib.call("jfb_mhd_convection", self._plan, *(t.data_ptr() for t in out),
                  self._stream())
        return out[:3], out[3:]


# reference name
PlaneCouetteMHDJax = PlaneCouetteMHD
