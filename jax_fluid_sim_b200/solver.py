"""Physics constants, state layout and state construction (reference-named API).

Mirrors ``HybridCompressibleSolver`` (hybrid/solver.py:12-470) and
``CompressibleStateLayout`` (hybrid/state.py:7-37) of superboss2300/jax-fluid-sim.
Pointwise conversions here are host/torch helpers for building states; the
flux arithmetic of the hot path lives in the CUDA kernels.
"""

from dataclasses import dataclass

import numpy as np
import torch

from .mesh import HybridMesh
from .reference import RefElement


@dataclass(frozen=True)
class CompressibleStateLayout:
    species_names: tuple = ()

    @property
    def number_of_variables(self):
        return 5 + len(self.species_names)

    @property
    def species(self):
        return slice(5, 5 + len(self.species_names))


class HybridCompressibleSolver:
    def __init__(self, mesh_path, species_names=(), gamma=1.4, gas_constant=1.0, polynomial_degree=2,
                 inviscid_flux="hllc", dynamic_viscosity=0.0, prandtl=0.72, use_wale=False, wale_constant=0.5,
                 turbulent_prandtl=0.9, chemistry_source=None):
        self.mesh = mesh_path if isinstance(mesh_path, HybridMesh) else HybridMesh(mesh_path)
        self.layout = CompressibleStateLayout(tuple(species_names))
        self.gamma = float(gamma)
        self.gas_constant = float(gas_constant)
        self.polynomial_degree = int(polynomial_degree)
        if inviscid_flux not in {"hllc", "rusanov"}:
            raise ValueError("inviscid_flux must be 'hllc' or 'rusanov'")
        if inviscid_flux != "hllc":
            raise NotImplementedError("the CUDA path implements the HLLC flux (the reference default)")
        if use_wale:
            raise NotImplementedError("WALE is not part of the CUDA path")
        if self.layout.number_of_variables not in (5, 16):
            raise NotImplementedError("the CUDA path supports 0 or 11 species")
        if self.polynomial_degree not in (1, 2, 3):
            raise ValueError("Only P1, P2, and P3 are currently implemented")
        self.inviscid_flux = inviscid_flux
        self.dynamic_viscosity = float(dynamic_viscosity)
        self.prandtl = float(prandtl)
        self.use_wale = False
        self.specific_heat_cp = self.gamma * self.gas_constant / (self.gamma - 1.0)
        self.thermal_conductivity = self.dynamic_viscosity * self.specific_heat_cp / self.prandtl
        self.reference_elements = {b.element_type: RefElement(b.element_type, self.polynomial_degree)
                                   for b in self.mesh.element_blocks}
        self.chemistry_source_function = chemistry_source

    # solver.py:63-81 (torch or numpy)
    def primitive_to_conserved(self, W):
        lib = torch if isinstance(W, torch.Tensor) else np
        rho = W[..., 0]
        vel = W[..., 1:4]
        E = W[..., 4] / (self.gamma - 1.0) + 0.5 * rho * (vel ** 2).sum(-1)
        parts = [rho[..., None], rho[..., None] * vel, E[..., None]]
        if self.layout.species_names:
            parts.append(rho[..., None] * W[..., 5:])
        return lib.concatenate(parts, -1) if lib is np else torch.cat(parts, -1)

    # solver.py:83-98
    def conserved_to_primitive(self, U):
        is_t = isinstance(U, torch.Tensor)
        rho = U[..., 0]
        srho = torch.clamp(rho, min=1e-14) if is_t else np.maximum(rho, 1e-14)
        vel = U[..., 1:4] / srho[..., None]
        ke = 0.5 * (U[..., 1:4] ** 2).sum(-1) / srho
        p = (self.gamma - 1.0) * (U[..., 4] - ke)
        parts = [rho[..., None], vel, p[..., None]]
        if self.layout.species_names:
            parts.append(U[..., 5:] / srho[..., None])
        return torch.cat(parts, -1) if is_t else np.concatenate(parts, -1)

    def uniform_state_blocks(self, density, velocity, pressure, mass_fractions=None, device="cuda"):
        """solver.py:421-455."""
        velocity = np.asarray(velocity, float)
        if velocity.shape != (3,):
            raise ValueError("velocity must have shape (3,)")
        prim = [density, *velocity, pressure]
        if self.layout.species_names:
            if mass_fractions is None:
                raise ValueError("Reacting layouts require mass_fractions")
            mf = np.asarray(mass_fractions, float)
            if mf.shape != (len(self.layout.species_names),):
                raise ValueError("mass_fractions has the wrong species count")
            if not np.isclose(mf.sum(), 1.0):
                raise ValueError("mass_fractions must sum to one")
            prim.extend(mf)
        prim = np.asarray(prim, float)
        out = {}
        for b in self.mesh.element_blocks:
            n = len(self.reference_elements[b.element_type].nodes)
            W = np.broadcast_to(prim, (len(b.connectivity), n, prim.size))
            out[b.element_type] = torch.as_tensor(self.primitive_to_conserved(W), device=device)
        return out

    def state_blocks_from_primitive_function(self, geometry_or_operator, function, device="cuda"):
        """solver.py:457-470: evaluate ``function(xyz) -> primitive`` at the solution nodes."""
        coords = geometry_or_operator.solution_node_coordinates
        out = {}
        for b in self.mesh.element_blocks:
            xyz = coords[b.element_type]
            W = np.asarray(function(xyz))
            expected = xyz.shape[:-1] + (self.layout.number_of_variables,)
            if W.shape != expected:
                raise ValueError(f"Primitive initializer returned {W.shape}; expected {expected} for {b.element_type}")
            out[b.element_type] = torch.as_tensor(self.primitive_to_conserved(W), device=device)
        return out
