"""Finite-rate Air-11 chemistry on the GPU: the reference's ``hybrid/chemistry`` API.

``ReactingFlowCoupler.react_block`` (``hybrid/chemistry/coupling.py:179-197``) advances
every node of an element block by one operator-split point-implicit chemistry step
(``integrator.py:31-104``) in one CUDA launch (``dgb_react_block``);
``Air11ParkMechanism.net_production_rates`` (``mechanism.py:159-220``) evaluates the
mass-action rates (``dgb_chem_rates``).  Single temperature only: the two-temperature
Landau-Teller relaxation (``relaxation.py``) is not implemented and passing one raises.
States are float64 CUDA tensors in the reference's layout (elements, nodes, 5 + species)
with the species partial densities from column 5 in the order e-, N+, O+, NO+, N2+, O2+,
N, O, NO, N2, O2.
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from .air11 import AIR11_REACTIONS, AIR11_SPECIES
from .mechanism import Reaction, Species, make_nasa7, mechanism_tables  # noqa: F401  (re-exported)


class ReactionMechanism:
    """A reaction mechanism (``hybrid/chemistry/mechanism.py:58-123``) built from ``Species``
    and ``Reaction`` records; its rates run on the GPU."""

    def __init__(self, species, reactions):
        self.species = tuple(species)
        self.reactions = tuple(reactions)
        self._init_tables(mechanism_tables(self.species, self.reactions))

    def _init_tables(self, t):
        self.species_names = tuple(sp.name for sp in self.species)
        self.num_species = len(self.species)
        self.num_reactions = len(self.reactions)
        self.molar_masses = np.asarray(t["molar_mass"], dtype=np.float64).copy()
        self._arrays = dict(
            molar_mass=N.as_f64(t["molar_mass"]),
            nu_forward=N.as_f64(t["nu_f"]),
            nu_reverse=N.as_f64(t["nu_r"]),
            efficiency=N.as_f64(t["alpha"]),
            arrhenius=N.as_f64(np.stack([t["A"], t["b"], t["theta"]], axis=1)),
            third_body=N.as_i32(t["third"]),
            forward_mode=N.as_i32(t["fmode"]),
            reverse_mode=N.as_i32(t["rmode"]),
            nasa_range=N.as_f64(t["trange"]),
            nasa_coeffs=N.as_f64(t["coeffs"]),
        )
        self._handle = None

    def descriptor(self):
        a = self._arrays
        m = N.ChemMechanism()
        m.num_species, m.num_reactions = self.num_species, self.num_reactions
        for name in ("molar_mass", "nu_forward", "nu_reverse", "efficiency", "arrhenius", "nasa_range",
                     "nasa_coeffs"):
            setattr(m, name, N.dptr(a[name]))
        for name in ("third_body", "forward_mode", "reverse_mode"):
            setattr(m, name, N.dptr(a[name], ctypes.c_int32))
        return m

    def _rates_handle(self):
        if self._handle is None:
            self._handle = _ChemHandle(self, N.ChemParams(0, 0, 300.0, 101325.0, 1.0, 1.4))
        return self._handle

    def net_production_rates(self, rho_species, T, Tv=None):
        """(omega_dot, w_dot) for rho_species (..., ns) and T (...) on the GPU."""
        omega, wdot, _ = self._rates(rho_species, T, Tv, jacobian=False)
        return omega, wdot

    def production_rate_jacobian(self, rho_species, T, Tv=None):
        """d w_dot / d rho_species (..., ns, ns): what ``integrator.py:78`` differentiates."""
        return self._rates(rho_species, T, Tv, jacobian=True)[2]

    def _rates(self, rho_species, T, Tv, jacobian):
        if Tv is not None and not torch.equal(torch.as_tensor(Tv), torch.as_tensor(T)):
            raise NotImplementedError("two-temperature rates (Tv != T) are not implemented")
        rho = _cuda_f64(rho_species)
        if rho.shape[-1] != self.num_species:
            raise ValueError(f"rho_species must end in {self.num_species} species")
        batch = rho.shape[:-1]
        Tt = torch.as_tensor(T, dtype=torch.float64, device=rho.device).expand(batch).contiguous()
        count = int(np.prod(batch)) if batch else 1
        omega = torch.empty_like(rho)
        wdot = torch.empty_like(rho)
        jac = torch.empty(batch + (self.num_species, self.num_species), dtype=torch.float64,
                          device=rho.device) if jacobian else None
        h = self._rates_handle()
        N.check(N.lib().dgb_chem_rates(h.ptr, rho.data_ptr(), Tt.data_ptr(), count, omega.data_ptr(),
                                       wdot.data_ptr(), jac.data_ptr() if jacobian else None, _stream(rho)))
        return omega, wdot, jac


class Air11ParkMechanism(ReactionMechanism):
    """The Air-11 Park mechanism (``hybrid/chemistry/air11_park.py:20-311``): 11 species,
    22 reactions, NASA-7 thermodynamics."""

    def __init__(self):
        super().__init__(AIR11_SPECIES, AIR11_REACTIONS)


class _ChemHandle:
    def __init__(self, mechanism, params):
        self.ptr = ctypes.c_void_p()
        L = N.lib()
        N.check(L.dgb_chem_create(ctypes.byref(mechanism.descriptor()), ctypes.byref(params),
                                  ctypes.byref(self.ptr)))
        self._destroy = L.dgb_chem_destroy      # kept: module globals may be gone at exit

    def __del__(self):
        ptr = getattr(self, "ptr", None)
        if ptr is not None and ptr.value:
            self._destroy(ptr)
            self.ptr = ctypes.c_void_p()


def _cuda_f64(x):
    t = torch.as_tensor(x)
    if not t.is_cuda:
        raise ValueError("chemistry runs on CUDA tensors (move the state to the GPU first)")
    return t.to(torch.float64).contiguous()


def _stream(t):
    return ctypes.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


class ReactingFlowCoupler:
    """Operator-split thermochemistry for element blocks (``coupling.py:19-209``).

    Same constructor arguments and defaults as the reference; the coupler scales by the
    freestream reference state when ``dimensionless`` (``coupling.py:55-67``).
    """

    def __init__(self, mechanism=None, relaxation=None, max_newton_iters=12, tolerance=1.0e-7,
                 dimensionless=False, reference_temperature=300.0, reference_pressure=101325.0,
                 reference_length=1.0, gamma=1.4):
        if relaxation is not None:
            raise NotImplementedError("two-temperature Landau-Teller relaxation is not implemented")
        self.mechanism = mechanism if mechanism is not None else Air11ParkMechanism()
        self.relaxation = None
        self.max_newton_iters = int(max_newton_iters)
        self.tolerance = float(tolerance)     # the reference never stops early on it either
        self.num_species = self.mechanism.num_species
        self.species_names = self.mechanism.species_names
        self.dimensionless = bool(dimensionless)
        self.gamma = float(gamma)
        self.T_ref = float(reference_temperature)
        self.p_ref = float(reference_pressure)
        self.L_ref = float(reference_length)
        R_univ = 8.31446261815324
        mean_mw = 1.0 / (0.767 / (2.0 * 0.0140067) + 0.233 / (2.0 * 0.015999))
        self.R_ref = R_univ / mean_mw
        self.rho_ref = self.p_ref / (self.R_ref * self.T_ref)
        self.u_ref = float(np.sqrt(self.R_ref * self.T_ref))
        self.e_ref = float(self.u_ref ** 2)
        self.t_ref = float(self.L_ref / self.u_ref)
        params = N.ChemParams(self.max_newton_iters, int(self.dimensionless), self.T_ref, self.p_ref, self.L_ref,
                              self.gamma)
        self._handle = _ChemHandle(self.mechanism, params)

    def react_block(self, U_block, dt, out=None):
        """Reacted copy of U_block (E, N, nvars); ``out`` may be U_block for an in-place update.
        ``dt`` is a float or a per-element array (E,) (local time stepping)."""
        U = U_block
        if not (isinstance(U, torch.Tensor) and U.is_cuda and U.dtype == torch.float64 and U.is_contiguous()):
            U = _cuda_f64(U_block)
        if U.dim() != 3:
            raise ValueError("U_block must be (elements, nodes, variables)")
        E, Np, nv = U.shape
        if nv < 5 + self.num_species:
            raise ValueError(f"State has {nv} variables; expected at least {5 + self.num_species} "
                             "for reacting mixture.")
        if out is None:
            out = torch.empty_like(U)
        elif out.shape != U.shape or out.dtype != torch.float64 or not out.is_contiguous() or not out.is_cuda:
            raise ValueError("out must be a contiguous float64 CUDA tensor shaped like U_block")
        dt_ptr, dt_val, keep = None, 0.0, None
        if isinstance(dt, (torch.Tensor, np.ndarray)) and np.ndim(dt) > 0:
            keep = torch.as_tensor(dt, dtype=torch.float64).to(U.device).reshape(-1).contiguous()
            if keep.numel() != E:
                raise ValueError("a per-element dt must hold one step per element")
            dt_ptr = keep.data_ptr()
        else:
            dt_val = float(dt)
        N.check(N.lib().dgb_react_block(self._handle.ptr, U.data_ptr(), out.data_ptr(), E, Np, nv, dt_val, dt_ptr,
                                        _stream(U)))
        return out

    def advance(self, states, dt):
        """``coupling.py:199-209``: react every block of a state dict."""
        return {name: self.react_block(block, dt) for name, block in states.items()}
