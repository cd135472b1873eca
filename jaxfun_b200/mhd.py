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
    rotational nonlinear form, Chebyshev family; ``precision`` "fp64", or
    "mixed" (complex64 periodic transforms and products of u, omega, b, j
    with the flow's base-flow terms added in FP64; FP64 operators, solves and
    state)."""

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
        precision: str = "fp64",
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
            precision=precision,
            device=device,
        )

    # imposed field and rotation rate (PlaneCouetteMRIShearpy sets them)
    background_b = (0.0, 0.0, 0.0)
    omega = 0.0

    def _create_plan(self, cfg: _lib.KMMConfig, handle: ctypes.c_void_p) -> None:
        prm = _lib.MHDParams()
        prm.eta = self.eta
        prm.omega = float(self.omega)
        for k in range(3):
            prm.b0[k] = float(self.background_b[k])
        _lib.call("jfb_mhd_create", ctypes.byref(cfg), ctypes.byref(prm), ctypes.byref(handle))

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
        out = self._fetch_mhd(min(2.0, hist + steps))
        self.check()
        return out

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


class PlaneCouetteMRIShearpy(PlaneCouetteMHD):
    """Rotating-shear plane-Couette MHD (pcf_mhd_mri_shearpy_jax.py:30-176):
    base flow U_b = -shear_rate x, Coriolis -2 omega e_z x u, imposed uniform
    field ``background_b`` in the Lorentz force and the EMF, nu = 1/Re,
    eta = 1/Rm.  The channel-mode seed of ``initial_state`` follows
    pcf_mhd_mri_shearpy_jax.py:99-147 (magnetic_seed "ax_yz" or
    "sinusoidal_bz_x")."""

    def __init__(
        self,
        N=(17, 16, 16),
        domain=((-1.0, 1.0), (0.0, 4.0 * math.pi), (0.0, 2.0 * math.pi)),
        Re: float = 400.0,
        Rm: float | None = None,
        omega: float = 1.0,
        shear_rate: float = 1.0,
        background_b=(0.0, 0.0, 0.025),
        dt: float = 0.01,
        family: str = "C",
        padding_factor=(1.0, 1.5, 1.5),
        perturbation_amplitude: float = 0.05,
        magnetic_amplitude: float = 0.0,
        magnetic_seed: str = "ax_yz",
        time_integrator: str | None = "SBDF3",
        nonlinear_form: str = "rotational",
        coefficient_path: str = "transform",
        solve_batching: str = "batched",
        precision: str = "fp64",
        device="cuda",
    ) -> None:
        from .kmm import KMM

        self.omega = float(omega)
        self.shear_rate = float(shear_rate)
        self.background_b = tuple(float(v) for v in background_b)
        if magnetic_seed not in {"ax_yz", "sinusoidal_bz_x"}:
            raise ValueError("magnetic_seed must be one of {ax_yz, sinusoidal_bz_x}")
        self.magnetic_seed = magnetic_seed
        self.Re = float(Re)
        self.U_wall = 1.0
        self.Rm = float(Re if Rm is None else Rm)
        self.eta = 1.0 / self.Rm
        self.magnetic_amplitude = float(magnetic_amplitude)
        self.perturbation_amplitude = float(perturbation_amplitude)
        KMM.__init__(
            self, N=N, domain=domain, nu=1.0 / self.Re, dt=dt, family=family,
            padding_factor=padding_factor, time_integrator=time_integrator,
            nonlinear_form=nonlinear_form, coefficient_path=coefficient_path,
            solve_batching=solve_batching, precision=precision, device=device,
            _u_wall=-self.shear_rate,
        )
        self.dUb_dx = -self.shear_rate

    def initial_state(self) -> MHDState:
        """The shearpy MRI channel-mode seed (pcf_mhd_mri_shearpy_jax.py:99-147)."""
        x, y, z = self.mesh()
        (a, b) = self.domain[0]
        xc, hw = 0.5 * (a + b), 0.5 * (b - a)
        wall = 1.0 - ((x - xc) / hw) ** 2
        amp = self.perturbation_amplitude
        Ly = self.domain[1][1] - self.domain[1][0]
        Lz = self.domain[2][1] - self.domain[2][0]
        ky, kz = 2.0 * math.pi / Ly, 2.0 * math.pi / Lz
        shape = self.N
        zero = torch.zeros(shape, dtype=torch.float64, device=self.device)
        u0, u1, u2 = zero, zero, zero
        if amp != 0.0:
            for h in (1, 2, 3):
                u0 = u0 + amp * wall * torch.cos(h * kz * z)
                u1 = u1 + amp * wall * torch.sin(h * kz * z)
            u0 = u0 + 0.1 * amp * wall * torch.sin(ky * y) * torch.cos(kz * z)
            u1 = u1 + 0.1 * amp * wall * torch.cos(ky * y) * torch.sin(kz * z)
            u2 = u2 + 0.1 * amp * wall * torch.sin(2.0 * ky * y) * torch.cos(2.0 * kz * z)
        flow = self.state_from_physical((u0, u1, u2))
        mag = self.magnetic_amplitude
        ax, ay, az = zero, zero, zero
        if mag != 0.0 and self.magnetic_seed == "ax_yz":
            ax = mag * wall * (1.0 / kz) * torch.sin(ky * y) * torch.sin(kz * z)
        elif mag != 0.0:
            xi = (x - xc) / hw
            ay = ay - (mag * hw / math.pi) * (torch.cos(math.pi * xi) + 1.0)
        A = self._A_state_from_physical((ax, ay, az))
        return self._ensure_mhd_history(MHDState(flow=flow, A=A))


class Ensemble:
    """Independent solvers (flow or MHD, any sizes) advanced together, one
    CUDA graph per step (``jfb_ensemble_*``): five launches per step over
    all members when every member is an MHD plan (``batched``), else every
    member on its own stream.  ``solve(states, steps)`` takes and returns
    one state per member."""

    def __init__(self, members) -> None:
        self.members = list(members)
        arr = (ctypes.c_void_p * len(self.members))(*(m._plan.value for m in self.members))
        handle = ctypes.c_void_p()
        _lib.call("jfb_ensemble_create", arr, len(self.members), ctypes.byref(handle))
        self._handle = handle
        b, n = ctypes.c_int32(), ctypes.c_int64()
        _lib.call("jfb_ensemble_info", handle, ctypes.byref(b), ctypes.byref(n))
        self.batched = bool(b.value)
        self.launches_per_step = int(n.value)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.load().jfb_ensemble_destroy(h)
            except Exception:
                pass
            self._handle = None

    def load(self, states) -> None:
        for m, st in zip(self.members, states, strict=True):
            m._load(st)

    def advance_resident(self, steps: int) -> None:
        stream = self.members[0]._stream()
        _lib.call("jfb_ensemble_advance", self._handle, int(steps), stream)
        for m in self.members:
            m._current = None

    def solve(self, states, steps: int):
        self.load(states)
        hist = [float(m._current.flow.history_steps if isinstance(m._current, MHDState)
                      else m._current.history_steps) for m in self.members]
        self.advance_resident(steps)
        out = []
        for m, h in zip(self.members, hist, strict=True):
            h = min(2.0, h + int(steps))
            out.append(m._fetch_mhd(h) if isinstance(m, PlaneCouetteMHD) else m._fetch(h))
        for m in self.members:
            m.check()
        return out


# reference names
PlaneCouetteMHDJax = PlaneCouetteMHD
PlaneCouetteMRIShearpyJax = PlaneCouetteMRIShearpy
