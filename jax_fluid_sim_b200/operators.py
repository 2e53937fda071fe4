"""DG spatial operators on the GPU (reference-named API).

``HybridEulerOperator`` and ``HybridNavierStokesOperator`` mirror
hybrid/spatial.py:10-249 and hybrid/navier_stokes.py:9-352 of
superboss2300/jax-fluid-sim: ``rhs``, ``inviscid_rhs`` and ``viscous_rhs`` take
a dict ``{element_type: (E, Np, nvars)}`` and an optional boundary descriptor
and return a new dict.  States are float64 CUDA tensors (numpy arrays are
copied to the device); all arithmetic runs in ``libdgb200.so``.
"""

import ctypes

import numpy as np
import torch

from . import _native as N
from .plan import Plan, block_affine_data, hex_affine_data, hex_sumfact_tables
from .reference import FACE_TYPE_ID, TYPE_ID


def _stream_ptr():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class NativePlan:
    """Owns one ``dgb_plan``: uploads the host plan tables and keeps the parameter block."""

    PRECISIONS = {"float64": 0, "mixed": 1}

    def __init__(self, plan: Plan, solver, viscous: bool, br2: float, sum_factorised=None, precision="float64",
                 affine=True, inverse_mass="device"):
        """``inverse_mass``: "device" builds the inverse mass matrices on the GPU from w|det J|
        (``dgb_plan_build_inverse_mass``); "host" uploads the host plan's copy (numpy), the
        set-up the device build is tested against."""
        if inverse_mass not in ("device", "host"):
            raise ValueError('inverse_mass must be "device" or "host"')
        L = N.lib()
        if precision not in self.PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(self.PRECISIONS)}")
        self.precision = precision
        self.plan = plan
        self.nblocks = len(plan.blocks)
        prm = N.Params()
        prm.degree = plan.degree
        prm.nvars = solver.layout.number_of_variables
        prm.num_blocks = self.nblocks
        prm.viscous = int(viscous)
        prm.gamma, prm.gas_constant = solver.gamma, solver.gas_constant
        prm.dynamic_viscosity, prm.thermal_conductivity = solver.dynamic_viscosity, solver.thermal_conductivity
        prm.br2_penalty = br2
        prm.has_boundary = 0
        prm.pos_density_floor = prm.pos_pressure_floor = 1e-10
        prm.pos_relative_floor = 0.05
        prm.adm_density_floor = prm.adm_pressure_floor = 1e-7
        prm.sensor_threshold = 5e-2
        prm.limiter = 0
        prm.precision = self.PRECISIONS[precision]
        self.params = prm
        handle = ctypes.c_void_p()
        N.check(L.dgb_plan_create(ctypes.byref(prm), ctypes.byref(handle)))
        self.handle = handle
        keep = []
        affine_counts = []
        single_hex = len(plan.blocks) == 1 and plan.blocks[0].etype == "hexahedron"
        if sum_factorised is None:
            sum_factorised = single_hex
        for b, bp in enumerate(plan.blocks):
            arrays = dict(basis=N.as_f64(bp.ref.B), basis_grad=N.as_f64(bp.ref.dB),
                          inv_jacobian=N.as_f64(bp.jinv), wdet=N.as_f64(bp.wdet),
                          length=N.as_f64(bp.length), face_sample_basis=N.as_f64(bp.face_sample_B),
                          p1_projector=N.as_f64(bp.p1_projector))
            if inverse_mass == "host":
                # the sum-factorised kernels stream M^-1 transposed (coalesced across nodes)
                arrays["inv_mass"] = N.as_f64(np.swapaxes(bp.minv, 1, 2) if sum_factorised else bp.minv)
            ef = N.as_i32(bp.elem_face)
            keep += list(arrays.values()) + [ef]
            d = N.BlockDesc(element_type=TYPE_ID[bp.etype], num_elements=bp.E, num_nodes=bp.Np, num_qp=bp.Nq,
                            num_local_faces=bp.nlf, elem_face=N.dptr(ef, ctypes.c_int32),
                            num_face_samples=len(bp.face_sample_B))
            for k, a in arrays.items():
                setattr(d, k, N.dptr(a))
            N.check(L.dgb_plan_set_block(handle, b, ctypes.byref(d)))
            if inverse_mass == "device":
                volume = N.as_f64(bp.volume)
                N.check(L.dgb_plan_build_inverse_mass(handle, b, N.dptr(volume), int(bool(sum_factorised))))
            if affine and not sum_factorised:
                aff, coef, ajinv, det, wref, mref_inv = block_affine_data(bp)
                aff = np.ascontiguousarray(aff, np.uint8)
                dbl = [N.as_f64(a) for a in (coef, ajinv, det, wref, mref_inv)]
                keep += [aff] + dbl
                N.check(L.dgb_plan_set_block_affine(handle, b, N.dptr(aff, ctypes.c_uint8), *[N.dptr(a) for a in dbl]))
                affine_counts.append(int(aff.sum()))
        for ftype, fp in plan.faces.items():
            ints = {k: N.as_i32(v) for k, v in dict(owner_block=fp.owner_block, owner_local=fp.owner_local,
                                                      owner_code=fp.ocode, nbr_block=fp.nbr_block,
                                                      nbr_local=fp.nbr_local, nbr_code=fp.ncode,
                                                      tags=fp.tags).items()}
            dbl = dict(normals=N.as_f64(fp.normals), weights=N.as_f64(fp.weights),
                       side_inv_jacobian=N.as_f64(fp.jinv_side))
            keep += list(ints.values()) + list(dbl.values())
            d = N.FaceDesc(face_type=FACE_TYPE_ID[ftype], num_faces=fp.F, num_qp=fp.nq)
            for k, a in ints.items():
                setattr(d, k, N.dptr(a, ctypes.c_int32))
            for k, a in dbl.items():
                setattr(d, k, N.dptr(a))
            N.check(L.dgb_plan_set_faces(handle, ctypes.byref(d)))
        for (etype, ftype), (B, dB) in plan.trace.items():
            B, dB = N.as_f64(B), N.as_f64(dB)
            keep += [B, dB]
            N.check(L.dgb_plan_set_trace(handle, TYPE_ID[etype], FACE_TYPE_ID[ftype], B.shape[0], B.shape[1],
                                         B.shape[2], N.dptr(B), N.dptr(dB)))
        if sum_factorised:
            if not single_hex:
                raise ValueError("the sum-factorised path needs a mesh of one hexahedron block")
            tables, lex, perm, nfq = hex_sumfact_tables(plan)
            tables, lex, perm = N.as_f64(tables), N.as_i32(lex), np.ascontiguousarray(perm, np.uint8)
            keep += [tables, lex, perm]
            N.check(L.dgb_plan_set_hex(handle, N.dptr(tables), N.dptr(lex, ctypes.c_int32), perm.shape[0], nfq,
                                       N.dptr(perm, ctypes.c_uint8)))
            if affine:
                aff, coef, ajinv, det = hex_affine_data(plan)
                aff, coef, ajinv, det = (np.ascontiguousarray(aff, np.uint8), N.as_f64(coef), N.as_f64(ajinv),
                                         N.as_f64(det))
                keep += [aff, coef, ajinv, det]
                N.check(L.dgb_plan_set_hex_affine(handle, N.dptr(aff, ctypes.c_uint8), N.dptr(coef), N.dptr(ajinv),
                                                  N.dptr(det)))
                self.affine_fraction = float(aff.mean())
                self.affine_count = int(aff.sum())
        if affine_counts:
            self.affine_count = sum(affine_counts)
            self.affine_fraction = self.affine_count / sum(bp.E for bp in plan.blocks)
            self.block_affine_counts = affine_counts
        self.sum_factorised = bool(sum_factorised)
        self.affine = bool(affine)
        N.check(L.dgb_plan_finalize(handle))
        self.fused = True          # the plan's default form of the hexahedron right-hand side
        self._pushed = self._snapshot()

    def enable_mood(self, coupling="reference", tables="device"):
        """Set up the MOOD subcell tables once (hybrid/subcell.py:442-471).  ``tables``: "device"
        builds them on the GPU from the reference subdivision and the geometry nodes
        (``dgb_plan_build_subcells``, ``dgb_plan_match_subcell_faces``); "host" uploads the
        host-built ``SubcellPlan`` (the construction the device build is tested against)."""
        if getattr(self, "mood_coupling", None) == coupling:
            return
        if getattr(self, "mood_coupling", None) is not None:
            raise ValueError("the subcell coupling of a plan is fixed once chosen")
        if tables not in ("device", "host"):
            raise ValueError('tables must be "device" or "host"')
        if tables == "device":
            self._build_mood_tables(coupling)
            return
        from .subcell import SubcellPlan
        L = N.lib()
        cache = self.plan.__dict__.setdefault("_subcell_plans", {})     # shared by plans of one mesh
        if coupling not in cache:
            cache[coupling] = SubcellPlan(self.plan.mesh, self.plan.degree, coupling)
        sp = cache[coupling]
        keep = []
        for b, (bp, sb) in enumerate(zip(self.plan.blocks, sp.blocks)):
            rs = sp.refs[bp.etype]
            gather, scatter = rs.coupling_indices(coupling)
            dbl = dict(projection=sb.projection, reconstruction=sb.reconstruction, volumes=sb.volumes,
                       centers=sb.centers, internal_normals=sb.internal_normals, internal_areas=sb.internal_areas,
                       boundary_normals=sb.boundary_normals, boundary_areas=sb.boundary_areas,
                       boundary_basis=sb.boundary_basis)
            ints = dict(internal_owner=rs.internal_owner, internal_neighbor=rs.internal_neighbor,
                        csr_ptr=rs.csr_ptr, csr_face=rs.csr_face, gather=gather, scatter=scatter)
            dbl = {k: N.as_f64(v) for k, v in dbl.items()}
            ints = {k: N.as_i32(v) for k, v in ints.items()}
            keep += list(dbl.values()) + list(ints.values())
            d = N.SubcellBlockDesc(num_subcells=rs.count, num_internal=len(rs.internal_faces),
                                   num_boundary=len(rs.boundary_faces))
            for k, a in dbl.items():
                setattr(d, k, N.dptr(a))
            for k, a in ints.items():
                setattr(d, k, N.dptr(a, ctypes.c_int32))
            N.check(L.dgb_plan_set_subcells(self.handle, b, ctypes.byref(d)))
        for ftype, (osub, nsub) in sp.faces.items():
            osub, nsub = N.as_i32(osub), N.as_i32(nsub)
            keep += [osub, nsub]
            N.check(L.dgb_plan_set_subcell_faces(self.handle, FACE_TYPE_ID[ftype], N.dptr(osub, ctypes.c_int32),
                                                 N.dptr(nsub, ctypes.c_int32)))
        N.check(L.dgb_plan_enable_mood(self.handle))
        self.mood_coupling = coupling
        self.subcell_plan = sp

    def _build_mood_tables(self, coupling):
        from .subcell import ReferenceSubcells, device_reference, subface_tables
        L = N.lib()
        mesh = self.plan.mesh
        refs = {b.element_type: ReferenceSubcells(b.element_type) for b in mesh.element_blocks}
        for b, (bp, block) in enumerate(zip(self.plan.blocks, mesh.element_blocks)):
            rs = refs[bp.etype]
            t, xyz = device_reference(mesh, block, self.plan.degree, rs)
            gather, scatter = rs.coupling_indices(coupling)
            dbl = {k: N.as_f64(t[k]) for k in ("rule_weights", "point_basis", "point_geometry_grad",
                                               "vertex_geometry", "boundary_basis")}
            ints = dict(cells=t["cells"], internal_faces=t["internal_faces"], boundary_faces=t["boundary_faces"],
                        internal_owner=rs.internal_owner, internal_neighbor=rs.internal_neighbor,
                        boundary_owner=rs.boundary_owner, csr_ptr=rs.csr_ptr, csr_face=rs.csr_face,
                        gather=gather, scatter=scatter)
            ints = {k: N.as_i32(v) for k, v in ints.items()}
            d = N.SubcellReference(num_subcells=rs.count, num_points=t["rule_weights"].shape[1],
                                   num_geometry_nodes=xyz.shape[1], num_vertices=len(rs.vertices),
                                   cell_size=rs.cells.shape[1], num_internal=len(rs.internal_faces),
                                   num_boundary=len(rs.boundary_faces))
            for k, a in dbl.items():
                setattr(d, k, N.dptr(a))
            for k, a in ints.items():
                setattr(d, k, N.dptr(a, ctypes.c_int32))
            N.check(L.dgb_plan_build_subcells(self.handle, b, ctypes.byref(d), N.dptr(N.as_f64(xyz))))
        for ftype, (osub, ncand) in subface_tables(mesh, refs).items():
            osub, ncand = N.as_i32(osub), N.as_i32(ncand)
            N.check(L.dgb_plan_match_subcell_faces(self.handle, FACE_TYPE_ID[ftype], N.dptr(osub, ctypes.c_int32),
                                                   N.dptr(ncand, ctypes.c_int32)))
        N.check(L.dgb_plan_enable_mood(self.handle))
        self.mood_coupling = coupling

    def set_tensor_cores(self, enable=True):
        """Run the inviscid volume integrals of the eligible dense blocks (prisms, tetrahedra up to
        P3) on the tensor cores (``dgb_plan_set_tensor_cores``); applies to mixed-precision plans
        without viscous terms.  Returns the number of blocks that use them."""
        n = ctypes.c_int(0)
        N.check(N.lib().dgb_plan_set_tensor_cores(self.handle, int(bool(enable)), ctypes.byref(n)))
        self.tensor_core_blocks = n.value
        return n.value

    def set_fused(self, enable=True):
        """Choose the three-launch (fused, the default) or the six-launch form of the
        sum-factorised hexahedron right-hand side (``dgb_plan_set_fused``)."""
        N.check(N.lib().dgb_plan_set_fused(self.handle, int(bool(enable))))
        self.fused = bool(enable)

    def device_errors(self, reset=True):
        """Error bits recorded on the device by kernels with bounded waits (0: none)."""
        out = ctypes.c_int(0)
        N.check(N.lib().dgb_plan_device_errors(self.handle, ctypes.byref(out), int(bool(reset))))
        return out.value

    def _snapshot(self):
        return bytes(self.params)

    def sync_params(self):
        snap = self._snapshot()
        if snap != self._pushed:
            N.check(N.lib().dgb_plan_update_params(self.handle, ctypes.byref(self.params)))
            self._pushed = snap

    def set_boundary(self, bc):
        if bc is None:
            self.params.has_boundary = 0
        else:
            bc.fill_params(self.params)
        self.sync_params()

    def state(self, blocks):
        st = N.State()
        for b, t in enumerate(blocks):
            st.block[b] = t.data_ptr() if t is not None else None
        return st

    def __del__(self):
        try:
            if getattr(self, "handle", None):
                N.lib().dgb_plan_destroy(self.handle)
                self.handle = None
        except Exception:
            pass


class HybridEulerOperator:
    """Anchor-form DG Euler residual (hybrid/spatial.py:10-249)."""

    _viscous = False

    def __init__(self, solver, br2_stabilization=None, sum_factorised=None, precision="float64", affine=True):
        """``precision``: "float64" (the reference's arithmetic) or "mixed" (float32 arithmetic in
        the trace, BR2-lift, volume and finalize kernels of every element type; the state, face
        fluxes, limiters, reductions and the stage update stay float64).  ``affine``: on the sum-factorised
        path, elements with an affine map use constant metrics and a tensor-product inverse mass
        matrix (equal to the dense one to round-off) instead of reading per-element tables."""
        self.solver = solver
        self.mesh = solver.mesh
        P = solver.polynomial_degree
        self.br2_stabilization = float((P + 1) * (P + 2) / 2 if br2_stabilization is None else br2_stabilization)
        self.plan = Plan(self.mesh, P)
        self.names = [b.element_type for b in self.mesh.element_blocks]
        viscous = self._viscous and solver.dynamic_viscosity > 0.0
        self.native = NativePlan(self.plan, solver, viscous, self.br2_stabilization, sum_factorised, precision,
                                 affine)
        self.precision = precision
        self.viscous = viscous
        self.solution_node_coordinates = {bp.etype: bp.node_xyz for bp in self.plan.blocks}

    def with_precision(self, precision):
        """The same operator (mesh, host tables, parameters) on a second device plan that runs in
        ``precision``; the host plan is shared, so this costs only the upload."""
        other = object.__new__(type(self))
        other.__dict__.update({k: v for k, v in self.__dict__.items() if k != "native"})
        other.native = NativePlan(self.plan, self.solver, self.viscous, self.br2_stabilization,
                                  self.native.sum_factorised, precision, self.native.affine)
        other.precision = precision
        return other

    # -- state plumbing
    def to_device(self, states):
        out = {}
        nv = self.solver.layout.number_of_variables
        for k, bp in zip(self.names, self.plan.blocks):
            t = states[k]
            if not isinstance(t, torch.Tensor):
                t = torch.as_tensor(np.asarray(t), device="cuda")
            if t.device.type != "cuda":
                t = t.cuda()
            t = t.to(torch.float64).contiguous()
            if tuple(t.shape) != (bp.E, bp.Np, nv):
                raise ValueError(f"{k} state has shape {tuple(t.shape)}; expected {(bp.E, bp.Np, nv)}")
            out[k] = t
        return out

    def _blocks(self, states):
        return [states[k] for k in self.names]

    def _run_rhs(self, states, boundary_state, want_inv, want_vis):
        U = self.to_device(states)
        self.native.set_boundary(boundary_state)
        inv = {k: torch.empty_like(U[k]) for k in self.names} if want_inv else None
        vis = {k: torch.empty_like(U[k]) for k in self.names} if want_vis else None
        s_in = self.native.state(self._blocks(U))
        s_inv = self.native.state(self._blocks(inv)) if inv else None
        s_vis = self.native.state(self._blocks(vis)) if vis else None
        N.check(N.lib().dgb_rhs(self.native.handle, ctypes.byref(s_in),
                                ctypes.byref(s_inv) if s_inv else None,
                                ctypes.byref(s_vis) if s_vis else None, _stream_ptr()))
        return inv, vis

    def rhs(self, states, boundary_state=None):
        inv, _ = self._run_rhs(states, boundary_state, True, False)
        return inv

    def autotune(self, states, boundary_state=None, reps=3):
        """Pick the threads-per-element width of the dense kernels by timing them on ``states``
        (dgb_plan_autotune); returns {kernel: {element_type: width}} (empty on the
        sum-factorised hexahedron path, whose launches are fixed)."""
        U = self.to_device(states)
        self.native.set_boundary(boundary_state)
        widths = np.zeros(3 * N.MAX_BLOCKS, np.int32)
        N.check(N.lib().dgb_plan_autotune(self.native.handle, ctypes.byref(self.native.state(self._blocks(U))),
                                          int(reps), N.dptr(widths, ctypes.c_int32), _stream_ptr()))
        out = {}
        for k, kernel in enumerate(("traces", "volume", "finalize")):
            row = {name: int(widths[k * N.MAX_BLOCKS + b]) for b, name in enumerate(self.names)
                   if widths[k * N.MAX_BLOCKS + b]}
            if row:
                out[kernel] = row
        return out

    def autotune_form(self, states, boundary_state=None, reps=3, mood=True):
        """Sum-factorised hexahedron path: time one right-hand side as an SSP-RK stage forms it
        (``dgb_rhs_profile_stage``, CUDA events around each launch) in the fused (three-launch) and
        in the six-launch form on ``states``, best of ``reps``, and keep the faster form in the plan.
        With ``mood`` the six-launch form keeps the viscous residual apart, as its MOOD step does;
        the fused form's MOOD step forms one residual and the viscous one for flagged elements only.
        Returns {"fused": ms, "six_launch": ms, "chosen": form}; an empty dict elsewhere."""
        if not self.native.sum_factorised:
            return {}
        U = self.to_device(states)
        self.native.set_boundary(boundary_state)
        st = self.native.state(self._blocks(U))
        ms = (ctypes.c_float * 6)()
        out = {}
        for name, fused in (("fused", True), ("six_launch", False)):
            self.native.set_fused(fused)
            split = int(bool(mood) and not fused and self.viscous)
            best = float("inf")
            for _ in range(int(reps) + 1):       # the first run loads the kernels
                N.check(N.lib().dgb_rhs_profile_stage(self.native.handle, ctypes.byref(st), split, ms,
                                                      _stream_ptr()))
                best = min(best, float(sum(ms)))
            out[name] = best
        out["chosen"] = "fused" if out["fused"] <= out["six_launch"] else "six_launch"
        self.native.set_fused(out["chosen"] == "fused")
        return out


class HybridNavierStokesOperator(HybridEulerOperator):
    """BR2 viscous operator on top of the Euler residual (hybrid/navier_stokes.py:9-352)."""

    _viscous = True

    def inviscid_rhs(self, states, boundary_state=None):
        inv, _ = self._run_rhs(states, boundary_state, True, False)
        return inv

    def viscous_rhs(self, states, boundary_state=None):
        if not self.viscous:
            U = self.to_device(states)
            return {k: torch.zeros_like(v) for k, v in U.items()}
        _, vis = self._run_rhs(states, boundary_state, False, True)
        return vis

    def rhs(self, states, boundary_state=None):
        if not self.viscous:
            return self.inviscid_rhs(states, boundary_state)
        inv, vis = self._run_rhs(states, boundary_state, True, True)
        return {k: inv[k] + vis[k] for k in inv}


def polynomial_br2_penalty(degree):
    """hybrid/navier_stokes.py:350-352."""
    return (degree + 1) * (degree + 2) / 2
