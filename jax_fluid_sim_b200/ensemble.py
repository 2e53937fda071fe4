"""Ensembles of independent cases advanced as one plan (no counterpart in the reference).

The cases' meshes are joined into one disjoint mesh (``meshgen.union``), so every RK stage is one
launch per kernel over all cases instead of one per case; each element carries its case id and
the kernels take the case's viscosity, conductivity, wall temperature and far-field state from
a table (``dgb_plan_set_cases``).  Everything else -- gamma, gas constant, degree, boundary tag
roles, limiter settings -- is shared, and one dt (the smallest stable one) serves all cases.
A case advanced inside the ensemble and the same case advanced alone with the same dt give the
same state: the element and face kernels see the same numbers.
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from . import meshgen
from .boundary import FarfieldWallBoundary
from .mesh import HybridMesh
from .operators import HybridNavierStokesOperator
from .solver import HybridCompressibleSolver


class HybridEnsemble:
    def __init__(self, sources, farfields, viscosities, polynomial_degree=2, gamma=1.4, gas_constant=1.0,
                 prandtl=0.72, wall_temperature=None, precision="float64"):
        """``sources``: one MeshSource per case (same physical names); ``farfields``: each case's
        far-field primitive state; ``viscosities``: each case's dynamic viscosity (> 0)."""
        if not (len(sources) == len(farfields) == len(viscosities)) or not sources:
            raise ValueError("one far-field state and one viscosity per mesh")
        viscosities = np.asarray(viscosities, np.float64)
        if np.any(viscosities <= 0.0):
            raise ValueError("ensemble cases need a positive viscosity")
        merged, counts = meshgen.union(sources)
        self.num_cases = len(sources)
        self.solver = HybridCompressibleSolver(HybridMesh(merged), gamma=gamma, gas_constant=gas_constant,
                                               polynomial_degree=polynomial_degree,
                                               dynamic_viscosity=float(viscosities[0]), prandtl=prandtl)
        self.operator = HybridNavierStokesOperator(self.solver, precision=precision)
        self.boundary = FarfieldWallBoundary(self.solver, farfields[0], wall_temperature=wall_temperature)
        nv = self.solver.layout.number_of_variables
        cp = gamma * gas_constant / (gamma - 1.0)
        table = np.zeros((self.num_cases, 3 + nv))
        table[:, 0] = viscosities
        table[:, 1] = viscosities * cp / prandtl
        table[:, 2] = 0.0 if wall_temperature is None else float(wall_temperature)
        table[:, 3:] = np.asarray(farfields, np.float64)
        self.table = table
        # element ranges of each case inside each block (the union lists cases in order)
        self.ranges = {}
        cases = []
        for bp in self.operator.plan.blocks:
            n = np.asarray([c.get(bp.etype, 0) for c in counts])
            ends = np.cumsum(n)
            self.ranges[bp.etype] = list(zip(ends - n, ends))
            cases.append(np.ascontiguousarray(np.repeat(np.arange(self.num_cases, dtype=np.int32), n)))
        self._case_ids = cases
        ptrs = (ctypes.c_void_p * len(cases))(*[c.ctypes.data for c in cases])
        t = N.as_f64(table)
        self._table = t
        N.check(N.lib().dgb_plan_set_cases(self.operator.native.handle, self.num_cases, N.dptr(t), ptrs))

    @property
    def dofs(self):
        return sum(bp.E * bp.Np for bp in self.operator.plan.blocks)

    def case_dofs(self, c):
        return sum((self.ranges[bp.etype][c][1] - self.ranges[bp.etype][c][0]) * bp.Np
                   for bp in self.operator.plan.blocks)

    def freestream_states(self, device="cuda"):
        """Every case at its own far-field state."""
        out = {}
        for bp in self.operator.plan.blocks:
            W = np.empty((bp.E, bp.Np, self.table.shape[1] - 3))
            for c, (a, b) in enumerate(self.ranges[bp.etype]):
                W[a:b] = self.table[c, 3:]
            out[bp.etype] = torch.as_tensor(self.solver.primitive_to_conserved(W), device=device)
        return out

    def split(self, states):
        """Per-case views {element_type: (E_c, Np, nvars)} of ensemble states."""
        return [{k: states[k][self.ranges[k][c][0]:self.ranges[k][c][1]] for k in states if
                 self.ranges[k][c][1] > self.ranges[k][c][0]} for c in range(self.num_cases)]
