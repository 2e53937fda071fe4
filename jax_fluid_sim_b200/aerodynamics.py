"""Aerodynamic forces and moments on wall boundaries (reference: hybrid/aerodynamics.py:13-305).

``AerodynamicForceCalculator`` keeps the reference's constructor and ``compute`` signature and
returns the same ``AerodynamicResult`` fields.  The surface integrals run on the GPU
(``dgb_wall_forces``): one right-hand-side evaluation fills the face traces, gradients and BR2
lifts, and one kernel integrates p n dA and -(tau . n) dA of the owner side over the wall faces
with their moments, reduced in a fixed order.  Only the 12 sums come back to the host.
"""

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _native as N
from .reference import FACE_TYPE_ID


@dataclass
class AerodynamicResult:
    step: int
    time: float
    Fx_total: float
    Fy_total: float
    Fz_total: float
    Fx_pressure: float
    Fy_pressure: float
    Fz_pressure: float
    Fx_viscous: float
    Fy_viscous: float
    Fz_viscous: float
    CD: float
    CD_p: float
    CD_f: float
    CL: float
    CL_p: float
    CL_f: float
    CS: float
    CS_p: float
    CS_f: float
    Mx: float
    My: float
    Mz: float
    CMx: float
    CMy: float
    CMz: float
    q_inf: float
    reference_area: float
    reference_length: float

    def summary_line(self) -> str:
        """aerodynamics.py:50-54."""
        return (f"C_D={self.CD:.4f} (p:{self.CD_p:.4f}, f:{self.CD_f:.4f}) "
                f"C_L={self.CL:+.4f} C_S={self.CS:+.4f}")


def face_points(plan):
    """Physical coordinates of every face point, {face type: (F, nq, 3)}, by the owner element's
    geometry map (the reference's face_metrics.physical_points)."""
    out = {}
    for ftype, fp in plan.faces.items():
        pts = np.empty((fp.F, fp.nq, 3))
        for b, block in enumerate(plan.mesh.element_blocks):
            sel = np.flatnonzero(fp.owner_block == b)
            if not len(sel):
                continue
            geo, xyz_b = plan.mesh.geometry(block)
            xyz = xyz_b[fp.owner_local[sel]]                                             # (f, n, 3)
            # the owner's reference face points are those of its trace code
            ref_pts = np.stack(plan.codes[(block.element_type, ftype)])                  # (codes, nq, 3)
            N1 = np.stack([geo.basis(r) for r in ref_pts])                               # (codes, nq, n)
            pts[sel] = np.einsum("fqk,fkd->fqd", N1[fp.ocode[sel]], xyz)
        out[ftype] = pts
    return out


class AerodynamicForceCalculator:
    def __init__(self, operator, boundary_state=None,
                 wall_tag_names=("sphere_wall", "cylinder_wall", "wall", "airfoil_wall"),
                 reference_area=None, reference_length=None, moment_center=(0.0, 0.0, 0.0)):
        """aerodynamics.py:60-111: wall tags by name (else the boundary's no-slip tags), and
        the reference length and area from the wall's bounding box unless given."""
        self.operator = operator
        self.solver = operator.solver
        self.boundary_state = boundary_state
        self.moment_center = np.asarray(moment_center, dtype=np.float64)
        names = self.solver.mesh.physical_names
        self.wall_tags = [int(names[n]) for n in wall_tag_names if n in names]
        if not self.wall_tags and hasattr(boundary_state, "no_slip_tags"):
            self.wall_tags = [int(t) for t in np.asarray(boundary_state.no_slip_tags)]
        if len(self.wall_tags) > N.MAX_TAGS:
            raise ValueError("at most 8 wall tags")
        plan = operator.plan
        pts = face_points(plan)
        self._points = {}
        coords = []
        for ftype, fp in plan.faces.items():
            p = N.as_f64(pts[ftype])
            self._points[ftype] = p
            N.check(N.lib().dgb_plan_set_face_points(operator.native.handle, FACE_TYPE_ID[ftype], N.dptr(p)))
            wall = (fp.nbr_block < 0) & np.isin(fp.tags, self.wall_tags)
            if np.any(wall):
                coords.append(pts[ftype][wall].reshape(-1, 3))
        if coords:
            allp = np.vstack(coords)
            lo, hi = allp.min(axis=0), allp.max(axis=0)
        else:
            lo, hi = np.full(3, -0.5), np.full(3, 0.5)
        dx, dy, dz = hi - lo
        diameter = max(dx, dy)
        self.reference_length = float(reference_length) if reference_length is not None else float(
            diameter if diameter > 0 else 1.0)
        if reference_area is not None:
            self.reference_area = float(reference_area)
        elif 0 < dz < 0.25 * min(dx, dy):
            self.reference_area = float(diameter * dz)       # extruded (quasi-2-D) body: D * span
        else:
            self.reference_area = float(np.pi * (0.5 * diameter) ** 2)
        self._tags = np.ascontiguousarray(self.wall_tags, np.int32)
        self._out = torch.zeros(12, dtype=torch.float64, device="cuda")

    def forces_device(self, states):
        """The 12 sums [F_p, M_p, F_v, M_v] as a device tensor (no host synchronisation)."""
        op = self.operator
        U = op.to_device(states)
        op.native.set_boundary(self.boundary_state)
        st = op.native.state(op._blocks(U))
        tags = self._tags if len(self._tags) else np.zeros(1, np.int32)
        N.check(N.lib().dgb_wall_forces(op.native.handle, ctypes.byref(st), N.dptr(tags, ctypes.c_int32),
                                        len(self._tags), N.dptr(self.moment_center),
                                        ctypes.c_void_p(self._out.data_ptr()),
                                        ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return self._out

    def compute(self, states, q_inf, step=0, current_time=0.0):
        """aerodynamics.py:149-305."""
        v = self.forces_device(states).cpu().numpy()
        F_p, M_p, F_v, M_v = v[0:3], v[3:6], v[6:9], v[9:12]
        F_t, M_t = F_p + F_v, M_p + M_v
        denom_force = max(q_inf * self.reference_area, 1.0e-14)
        denom_moment = max(denom_force * self.reference_length, 1.0e-14)
        c_p, c_f = F_p / denom_force, F_v / denom_force
        return AerodynamicResult(
            step=step, time=current_time,
            Fx_total=float(F_t[0]), Fy_total=float(F_t[1]), Fz_total=float(F_t[2]),
            Fx_pressure=float(F_p[0]), Fy_pressure=float(F_p[1]), Fz_pressure=float(F_p[2]),
            Fx_viscous=float(F_v[0]), Fy_viscous=float(F_v[1]), Fz_viscous=float(F_v[2]),
            CD=float(c_p[0] + c_f[0]), CD_p=float(c_p[0]), CD_f=float(c_f[0]),
            CL=float(c_p[1] + c_f[1]), CL_p=float(c_p[1]), CL_f=float(c_f[1]),
            CS=float(c_p[2] + c_f[2]), CS_p=float(c_p[2]), CS_f=float(c_f[2]),
            Mx=float(M_t[0]), My=float(M_t[1]), Mz=float(M_t[2]),
            CMx=float(M_t[0] / denom_moment), CMy=float(M_t[1] / denom_moment), CMz=float(M_t[2] / denom_moment),
            q_inf=float(q_inf), reference_area=self.reference_area, reference_length=self.reference_length)
