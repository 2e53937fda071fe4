"""SSP-RK3 time integration on the GPU (reference-named API).

Mirrors ``HybridSSPRK3`` (hybrid/time_integration.py:8-671) of
superboss2300/jax-fluid-sim: ``stable_dt``, ``state_admissibility`` and
``checked_step``.  A checked step is one native call that runs the three
Shu-Osher stages -- each a fused RHS + blend kernel sequence, the positivity
limiter and the admissibility reduction -- and leaves (valid, rho_min, p_min)
in a device status word that the host reads once per step.
"""

import ctypes

import torch

from . import _native as N
from .limiter import HybridMOODSubcellLimiter, HybridPositivityLimiter
from .operators import _stream_ptr


class HybridSSPRK3:
    def __init__(self, operator, cfl=0.15, limiter=None, density_floor=1.0e-7, pressure_floor=1.0e-7,
                 maximum_rejections=16, graph=False):
        """``graph=True`` runs every checked step as one CUDA graph (captured on the first step and
        again whenever the state buffers, dt or the plan's parameters change)."""
        self.operator = operator
        self.graph = bool(graph)
        self.solver = operator.solver
        self.cfl = float(cfl)
        self.limiter = limiter
        self.density_floor = float(density_floor)
        self.pressure_floor = float(pressure_floor)
        self.maximum_rejections = int(maximum_rejections)
        self._status = torch.zeros(3, dtype=torch.float64, device="cuda")   # dgb_status (24 bytes)
        self._dt = torch.zeros(1, dtype=torch.float64, device="cuda")
        if limiter is not None and not isinstance(limiter, (HybridPositivityLimiter, HybridMOODSubcellLimiter)):
            raise NotImplementedError("supported stage limiters: HybridPositivityLimiter, HybridMOODSubcellLimiter")

    @property
    def characteristic_lengths(self):
        return {bp.etype: bp.length for bp in self.operator.plan.blocks}

    def _configure(self, boundary_state):
        native = self.operator.native
        prm = native.params
        prm.adm_density_floor = self.density_floor
        prm.adm_pressure_floor = self.pressure_floor
        if isinstance(self.limiter, HybridMOODSubcellLimiter):
            self.limiter.configure(prm)
            prm.limiter = 2
        elif isinstance(self.limiter, HybridPositivityLimiter):
            self.limiter.configure(prm)
            prm.limiter = 1
        else:
            prm.limiter = 0
        native.set_boundary(boundary_state)

    def stable_dt_device(self, states, boundary_state=None):
        """dt as a device tensor (no host synchronisation)."""
        op = self.operator
        U = op.to_device(states)
        self._configure(boundary_state)
        st = op.native.state(op._blocks(U))
        N.check(N.lib().dgb_stable_dt(op.native.handle, ctypes.byref(st), self.cfl,
                                      ctypes.c_void_p(self._dt.data_ptr()), _stream_ptr()))
        return self._dt

    def stable_dt(self, states, boundary_state=None):
        return float(self.stable_dt_device(states, boundary_state).item())

    def _status_tuple(self):
        raw = self._status.cpu()
        valid = bool(raw.view(torch.int32)[0].item())
        return valid, float(raw[1]), float(raw[2])

    def state_admissibility(self, states):
        op = self.operator
        U = op.to_device(states)
        self._configure(None)
        st = op.native.state(op._blocks(U))
        N.check(N.lib().dgb_admissibility(op.native.handle, ctypes.byref(st),
                                          ctypes.c_void_p(self._status.data_ptr()), _stream_ptr()))
        return self._status_tuple()

    def checked_step_inplace(self, states, dt, boundary_state=None):
        """Advance device states in place; returns the device status tensor (no sync)."""
        op = self.operator
        self._configure(boundary_state)
        st = op.native.state(op._blocks(states))
        step = N.lib().dgb_ssprk3_step_graph if self.graph else N.lib().dgb_ssprk3_step
        N.check(step(op.native.handle, ctypes.byref(st), float(dt), ctypes.c_void_p(self._status.data_ptr()),
                     _stream_ptr()))
        return self._status

    def checked_step(self, states, dt, boundary_state=None):
        """time_integration.py:441-583 (non-MOOD branch): returns (states, valid, rho_min, p_min)."""
        if isinstance(dt, dict):
            raise NotImplementedError("local time stepping is outside the CUDA path")
        U = {k: v.clone() for k, v in self.operator.to_device(states).items()}
        self.checked_step_inplace(U, dt, boundary_state)
        valid, rmin, pmin = self._status_tuple()
        return U, valid, rmin, pmin
