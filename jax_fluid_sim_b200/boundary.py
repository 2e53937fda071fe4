"""Boundary descriptor (reference: ``FarfieldWallBoundary``, hybrid/boundary.py:6-102).

In the reference the boundary object is a Python callable evaluated inside the
residual.  Here it is a descriptor -- physical tags grouped by role, the
far-field primitive state and the wall temperature -- that the CUDA kernels
evaluate per face point with the same rules: walls reflect the normal
velocity, inlets impose the far-field state, everything else (outlets, unknown
tags) copies the interior; the viscous ghost negates velocity on no-slip walls
and sets T = 2 T_wall - T when a wall temperature is given.
"""

import numpy as np


class FarfieldWallBoundary:
    def __init__(self, solver, farfield_primitive, inlet_names=("inlet",), outlet_names=("outlet",),
                 wall_names=("walls", "sphere_wall", "cylinder_wall", "airfoil_wall", "symmetry"),
                 no_slip_names=("sphere_wall", "cylinder_wall", "airfoil_wall"),
                 slip_names=("walls", "symmetry"), wall_temperature=None):
        self.solver = solver
        self.wall_temperature = None if wall_temperature is None else float(wall_temperature)
        self.farfield_primitive = np.asarray(farfield_primitive, np.float64)
        if self.farfield_primitive.shape != (solver.layout.number_of_variables,):
            raise ValueError("farfield_primitive has the wrong state size")
        names = solver.mesh.physical_names

        def tags(group):
            return np.asarray([names[n] for n in group if n in names], np.int32)

        self.inlet_tags, self.outlet_tags = tags(inlet_names), tags(outlet_names)
        self.wall_tags, self.no_slip_tags, self.slip_tags = tags(wall_names), tags(no_slip_names), tags(slip_names)
        for group in (self.inlet_tags, self.wall_tags, self.no_slip_tags, self.slip_tags):
            if len(group) > 8:
                raise ValueError("at most 8 physical tags per boundary role")

    @staticmethod
    def _matches(tags, choices):
        tags = np.asarray(tags)
        if choices.size == 0:
            return np.zeros(tags.shape, bool)
        return np.any(tags[..., None] == choices, axis=-1)

    def fill_params(self, prm):
        prm.has_boundary = 1
        for v, x in enumerate(self.farfield_primitive):
            prm.farfield_primitive[v] = float(x)
        for field, group in (("inlet", self.inlet_tags), ("wall", self.wall_tags),
                             ("no_slip", self.no_slip_tags), ("slip", self.slip_tags)):
            arr = getattr(prm, f"{field}_tags")
            for k, t in enumerate(group):
                arr[k] = int(t)
            setattr(prm, f"n_{field}", len(group))
        prm.has_wall_temperature = int(self.wall_temperature is not None)
        prm.wall_temperature = 0.0 if self.wall_temperature is None else self.wall_temperature
