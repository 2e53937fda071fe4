"""Positivity limiter, troubled-cell sensor and MOOD detection on the GPU.

Mirror ``HybridPositivityLimiter`` (hybrid/limiter.py:11-147),
``HybridTroubledCellSensor`` (:150-185) and ``HybridMOODSubcellLimiter.troubled``
(:285-300) of superboss2300/jax-fluid-sim.  Each call runs one element-parallel
kernel of ``libdgb200.so`` over every block.
"""

import ctypes

import torch

from . import _native as N
from .operators import _stream_ptr


class HybridPositivityLimiter:
    def __init__(self, operator, density_floor=1.0e-10, pressure_floor=1.0e-10, relative_floor=0.05):
        self.operator = operator
        self.solver = operator.solver
        self.density_floor = float(density_floor)
        self.pressure_floor = float(pressure_floor)
        self.relative_floor = float(relative_floor)

    def configure(self, params):
        params.pos_density_floor = self.density_floor
        params.pos_pressure_floor = self.pressure_floor
        params.pos_relative_floor = self.relative_floor

    def __call__(self, states):
        op = self.operator
        U = {k: v.clone() for k, v in op.to_device(states).items()}
        self.configure(op.native.params)
        op.native.sync_params()
        st = op.native.state(op._blocks(U))
        N.check(N.lib().dgb_positivity(op.native.handle, ctypes.byref(st), _stream_ptr()))
        return U


class HybridTroubledCellSensor:
    def __init__(self, operator, threshold=5.0e-2):
        self.operator = operator
        self.solver = operator.solver
        self.threshold = float(threshold)

    def _run(self, states, positivity=None):
        op = self.operator
        U = op.to_device(states)
        op.native.params.sensor_threshold = self.threshold
        if positivity is not None:
            positivity.configure(op.native.params)
        op.native.sync_params()
        sens = {k: torch.empty(v.shape[0], dtype=torch.float64, device="cuda") for k, v in U.items()}
        flags = {k: torch.empty(v.shape[0], dtype=torch.uint8, device="cuda") for k, v in U.items()}
        sp = (ctypes.c_void_p * N.MAX_BLOCKS)(*[sens[k].data_ptr() for k in op.names])
        fp = (ctypes.c_void_p * N.MAX_BLOCKS)(*[flags[k].data_ptr() for k in op.names])
        st = op.native.state(op._blocks(U))
        N.check(N.lib().dgb_troubled(op.native.handle, ctypes.byref(st), sp, fp, _stream_ptr()))
        return sens, flags

    def __call__(self, states):
        """(sensor values, sensor > threshold) per block; the flags here are the sensor only."""
        sens, _ = self._run(states)
        return sens, {k: v > self.threshold for k, v in sens.items()}


RECONSTRUCTIONS = {"constant": 0, "tvd": 1, "weno": 2}


class HybridSubcellFV:
    """Conservative subcell FV recompute (hybrid/subcell.py:442-950) on the GPU.

    ``coupling="reference"`` reproduces the reference's DG-FV coupling indices exactly
    (see jax_fluid_sim_b200/subcell.py); ``coupling="subcell"`` couples each boundary
    subface to the subcell that owns it."""

    def __init__(self, operator, division_count=4, reconstruction="weno", coupling="reference"):
        if division_count != 4:
            raise ValueError("P2 subcell coupling currently requires division_count=4")
        if reconstruction not in RECONSTRUCTIONS:
            raise ValueError(f"Unknown subcell reconstruction mode: {reconstruction!r}")
        self.operator = operator
        self.reconstruction = reconstruction
        operator.native.enable_mood(coupling)

    def recompute(self, states, dg_candidate, dt, troubled, boundary_state=None, additional_rhs=None):
        op = self.operator
        base, cand = op.to_device(states), op.to_device(dg_candidate)
        arhs = op.to_device(additional_rhs) if additional_rhs is not None else None
        if isinstance(dt, dict):
            raise NotImplementedError("local time stepping is outside the CUDA path")
        flags = {k: torch.as_tensor(troubled[k], device="cuda").to(torch.uint8).contiguous() for k in op.names}
        op.native.params.reconstruction = RECONSTRUCTIONS[self.reconstruction]
        op.native.set_boundary(boundary_state)
        out = {k: torch.empty_like(v) for k, v in base.items()}
        fp = (ctypes.c_void_p * N.MAX_BLOCKS)(*[flags[k].data_ptr() for k in op.names])
        sb, sc, so = (op.native.state(op._blocks(x)) for x in (base, cand, out))
        sa = op.native.state(op._blocks(arhs)) if arhs is not None else None
        N.check(N.lib().dgb_subcell_recompute(op.native.handle, ctypes.byref(sb), ctypes.byref(sc), float(dt),
                                              ctypes.byref(sa) if sa is not None else None, fp,
                                              ctypes.byref(so), _stream_ptr()))
        return out


class HybridMOODSubcellLimiter:
    """A-posteriori P-DG / subcell-FV recomputation (hybrid/limiter.py:267-343)."""

    def __init__(self, operator, threshold=5.0e-2, positivity=None, reconstruction="weno", coupling="reference"):
        self.operator = operator
        self.sensor = HybridTroubledCellSensor(operator, threshold)
        self.positivity = HybridPositivityLimiter(operator) if positivity is None else positivity
        self.reconstruction = reconstruction
        self.subcell = HybridSubcellFV(operator, reconstruction=reconstruction, coupling=coupling)

    def configure(self, params):
        self.positivity.configure(params)
        params.sensor_threshold = self.sensor.threshold
        params.reconstruction = RECONSTRUCTIONS[self.reconstruction]

    def troubled(self, candidate):
        _, flags = self.sensor._run(candidate, self.positivity)
        return {k: v.bool() for k, v in flags.items()}

    def recompute(self, base, dg_candidate, dt, boundary_state=None, additional_rhs=None, detection_state=None,
                  troubled_mask=None):
        troubled = troubled_mask if troubled_mask is not None else self.troubled(
            dg_candidate if detection_state is None else detection_state)
        corrected = self.subcell.recompute(base, dg_candidate, dt, troubled, boundary_state, additional_rhs)
        return self.positivity(corrected)

    def __call__(self, states):
        return self.positivity(states)
