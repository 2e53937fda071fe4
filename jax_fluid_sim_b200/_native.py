"""ctypes binding of ``libdgb200.so`` (declarations in ``include/dgb200.h``).

There is no CPU fallback: if the library cannot be loaded, every entry point
raises.  PyTorch is used only for device allocations and streams; the library
receives raw pointers.
"""

import ctypes
from pathlib import Path

import numpy as np

MAX_BLOCKS, MAX_TAGS, MAX_VARS = 3, 8, 16
LIB_PATH = Path(__file__).resolve().parent / "libdgb200.so"

c_int, c_double, c_void_p = ctypes.c_int, ctypes.c_double, ctypes.c_void_p
P_double = ctypes.POINTER(ctypes.c_double)
P_int32 = ctypes.POINTER(ctypes.c_int32)
P_int64 = ctypes.POINTER(ctypes.c_int64)


class Params(ctypes.Structure):
    _fields_ = [
        ("degree", c_int), ("nvars", c_int), ("num_blocks", c_int), ("viscous", c_int),
        ("gamma", c_double), ("gas_constant", c_double), ("dynamic_viscosity", c_double),
        ("thermal_conductivity", c_double), ("br2_penalty", c_double),
        ("has_boundary", c_int),
        ("farfield_primitive", c_double * MAX_VARS),
        ("inlet_tags", c_int * MAX_TAGS), ("n_inlet", c_int),
        ("wall_tags", c_int * MAX_TAGS), ("n_wall", c_int),
        ("no_slip_tags", c_int * MAX_TAGS), ("n_no_slip", c_int),
        ("slip_tags", c_int * MAX_TAGS), ("n_slip", c_int),
        ("has_wall_temperature", c_int), ("wall_temperature", c_double),
        ("pos_density_floor", c_double), ("pos_pressure_floor", c_double), ("pos_relative_floor", c_double),
        ("adm_density_floor", c_double), ("adm_pressure_floor", c_double),
        ("sensor_threshold", c_double),
        ("limiter", c_int),
        ("reconstruction", c_int),
        ("precision", c_int),
    ]


class SubcellBlockDesc(ctypes.Structure):
    _fields_ = [
        ("num_subcells", c_int), ("num_internal", c_int), ("num_boundary", c_int),
        ("projection", P_double), ("reconstruction", P_double), ("volumes", P_double), ("centers", P_double),
        ("internal_normals", P_double), ("internal_areas", P_double), ("boundary_normals", P_double),
        ("boundary_areas", P_double), ("internal_owner", P_int32), ("internal_neighbor", P_int32),
        ("csr_ptr", P_int32), ("csr_face", P_int32), ("boundary_basis", P_double), ("gather", P_int32),
        ("scatter", P_int32),
    ]


class SubcellReference(ctypes.Structure):
    _fields_ = [
        ("num_subcells", c_int), ("num_points", c_int), ("num_geometry_nodes", c_int), ("num_vertices", c_int),
        ("cell_size", c_int), ("num_internal", c_int), ("num_boundary", c_int),
        ("rule_weights", P_double), ("point_basis", P_double), ("point_geometry_grad", P_double),
        ("vertex_geometry", P_double), ("cells", P_int32), ("internal_faces", P_int32), ("boundary_faces", P_int32),
        ("internal_owner", P_int32), ("internal_neighbor", P_int32), ("boundary_owner", P_int32),
        ("csr_ptr", P_int32), ("csr_face", P_int32), ("boundary_basis", P_double), ("gather", P_int32),
        ("scatter", P_int32),
    ]


class BlockDesc(ctypes.Structure):
    _fields_ = [
        ("element_type", c_int), ("num_elements", c_int), ("num_nodes", c_int), ("num_qp", c_int),
        ("num_local_faces", c_int),
        ("basis", P_double), ("basis_grad", P_double), ("inv_jacobian", P_double), ("wdet", P_double),
        ("inv_mass", P_double), ("elem_face", P_int32), ("length", P_double),
        ("num_face_samples", c_int), ("face_sample_basis", P_double), ("p1_projector", P_double),
    ]


class FaceDesc(ctypes.Structure):
    _fields_ = [
        ("face_type", c_int), ("num_faces", c_int), ("num_qp", c_int),
        ("owner_block", P_int32), ("owner_local", P_int32), ("owner_code", P_int32),
        ("nbr_block", P_int32), ("nbr_local", P_int32), ("nbr_code", P_int32),
        ("tags", P_int32), ("normals", P_double), ("weights", P_double), ("side_inv_jacobian", P_double),
    ]


class State(ctypes.Structure):
    _fields_ = [("block", c_void_p * MAX_BLOCKS)]


class Status(ctypes.Structure):
    _fields_ = [("valid", ctypes.c_int32), ("pad", ctypes.c_int32), ("rho_min", c_double), ("p_min", c_double)]


class ChemMechanism(ctypes.Structure):
    _fields_ = [("num_species", c_int), ("num_reactions", c_int), ("molar_mass", P_double),
                ("nu_forward", P_double), ("nu_reverse", P_double), ("efficiency", P_double),
                ("arrhenius", P_double), ("third_body", P_int32), ("forward_mode", P_int32),
                ("reverse_mode", P_int32), ("nasa_range", P_double), ("nasa_coeffs", P_double)]


class ChemParams(ctypes.Structure):
    _fields_ = [("max_newton_iters", c_int), ("dimensionless", c_int), ("reference_temperature", c_double),
                ("reference_pressure", c_double), ("reference_length", c_double), ("gamma", c_double)]


_lib = None


def lib():
    """Load the library once; raise loudly when it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m jax_fluid_sim_b200.build`")
        L = ctypes.CDLL(str(LIB_PATH))
        L.dgb_last_error.restype = ctypes.c_char_p
        L.dgb_noalloc_last_error.restype = ctypes.c_char_p
        L.dgb_stable_dt_noalloc.argtypes = [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_double, c_double,
                                            c_double, c_double, c_double, c_double, c_void_p, c_void_p]
        L.dgb_stable_dt_noalloc.restype = c_int
        L.dgb_version.restype = c_int
        sigs = {
            "dgb_plan_create": [ctypes.POINTER(Params), ctypes.POINTER(c_void_p)],
            "dgb_plan_set_block": [c_void_p, c_int, ctypes.POINTER(BlockDesc)],
            "dgb_plan_set_faces": [c_void_p, ctypes.POINTER(FaceDesc)],
            "dgb_plan_set_trace": [c_void_p, c_int, c_int, c_int, c_int, c_int, P_double, P_double],
            "dgb_plan_finalize": [c_void_p],
            "dgb_plan_set_hex": [c_void_p, P_double, P_int32, c_int, c_int, ctypes.POINTER(ctypes.c_uint8)],
            "dgb_plan_set_hex_affine": [c_void_p, ctypes.POINTER(ctypes.c_uint8), P_double, P_double, P_double],
            "dgb_plan_set_face_points": [c_void_p, c_int, P_double],
            "dgb_raster_render": [ctypes.POINTER(RasterDesc), ctypes.POINTER(State), c_int, ctypes.c_double, c_int,
                                  ctypes.c_double, ctypes.c_double, c_void_p, c_void_p, c_void_p],
            "dgb_wall_forces": [c_void_p, ctypes.POINTER(State), P_int32, c_int, P_double, c_void_p, c_void_p],
            "dgb_plan_autotune": [c_void_p, ctypes.POINTER(State), c_int, P_int32, c_void_p],
            "dgb_plan_set_tensor_cores": [c_void_p, c_int, ctypes.POINTER(c_int)],
            "dgb_plan_set_fused": [c_void_p, c_int],
            "dgb_plan_device_errors": [c_void_p, ctypes.POINTER(c_int), c_int],
            "dgb_plan_set_cases": [c_void_p, c_int, P_double, ctypes.POINTER(ctypes.c_void_p)],
            "dgb_plan_set_block_affine": [c_void_p, c_int, ctypes.POINTER(ctypes.c_uint8), P_double, P_double,
                                          P_double, P_double, P_double],
            "dgb_plan_build_inverse_mass": [c_void_p, c_int, P_double, c_int],
            "dgb_spd_inverse": [c_void_p, c_int, c_int, c_void_p, c_void_p],
            "dgb_subcell_face_metrics": [P_double, c_int, c_int, P_int32, P_int32, c_int, P_double, c_int, P_int32,
                                         P_int32, P_double, P_double, P_double],
            "dgb_affine_test": [P_double, c_int, c_int, c_double, ctypes.POINTER(ctypes.c_uint8), P_double],
            "dgb_pair_faces": [P_int64, c_int, ctypes.c_int64, P_int64, P_int64, P_int64, P_int64],
            "dgb_msh2_nodes": [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, P_int64, P_double],
            "dgb_msh2_elements": [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, P_int32, P_int32, P_int64,
                                  P_int64, ctypes.c_int64],
            "dgb_msh4_nodes": [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, P_int64, P_double],
            "dgb_msh4_elements": [ctypes.c_char_p, ctypes.c_int64, ctypes.c_int64, P_int32, P_int32, P_int32,
                                  P_int64, P_int64, ctypes.c_int64],
            "dgb_map_metrics": [P_double, P_int32, c_int, c_int, P_double, c_int, P_double, P_double, P_double,
                                P_double, P_double, P_double, P_double, P_double, P_double],
            "dgb_plan_destroy": [c_void_p],
            "dgb_plan_update_params": [c_void_p, ctypes.POINTER(Params)],
            "dgb_rhs": [c_void_p, ctypes.POINTER(State), ctypes.POINTER(State), ctypes.POINTER(State), c_void_p],
            "dgb_stable_dt": [c_void_p, ctypes.POINTER(State), c_double, c_void_p, c_void_p],
            "dgb_positivity": [c_void_p, ctypes.POINTER(State), c_void_p],
            "dgb_troubled": [c_void_p, ctypes.POINTER(State), c_void_p, c_void_p, c_void_p],
            "dgb_admissibility": [c_void_p, ctypes.POINTER(State), c_void_p, c_void_p],
            "dgb_ssprk3_step": [c_void_p, ctypes.POINTER(State), c_double, c_void_p, c_void_p],
            "dgb_ssprk3_step_graph": [c_void_p, ctypes.POINTER(State), c_double, c_void_p, c_void_p],
            "dgb_rhs_profile": [c_void_p, ctypes.POINTER(State), ctypes.POINTER(ctypes.c_float), c_void_p],
            "dgb_rhs_profile_stage": [c_void_p, ctypes.POINTER(State), c_int, ctypes.POINTER(ctypes.c_float),
                                      c_void_p],
            "dgb_plan_set_subcells": [c_void_p, c_int, ctypes.POINTER(SubcellBlockDesc)],
            "dgb_plan_set_subcell_faces": [c_void_p, c_int, P_int32, P_int32],
            "dgb_plan_build_subcells": [c_void_p, c_int, ctypes.POINTER(SubcellReference), P_double],
            "dgb_plan_match_subcell_faces": [c_void_p, c_int, P_int32, P_int32],
            "dgb_plan_enable_mood": [c_void_p],
            "dgb_chem_create": [ctypes.POINTER(ChemMechanism), ctypes.POINTER(ChemParams), ctypes.POINTER(c_void_p)],
            "dgb_chem_destroy": [c_void_p],
            "dgb_react_block": [c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_int, c_int, c_double, c_void_p,
                                c_void_p],
            "dgb_chem_rates": [c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p, c_void_p, c_void_p],
            "dgb_subcell_recompute": [c_void_p, ctypes.POINTER(State), ctypes.POINTER(State), c_double,
                                      ctypes.POINTER(State), c_void_p, ctypes.POINTER(State), c_void_p],
        }
        for name, args in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = c_int
        _lib = L
    return _lib


def check(rc):
    if rc != 0:
        msg = lib().dgb_last_error().decode()
        if rc == -1:
            raise ValueError(msg)
        if rc == -3:
            raise NotImplementedError(msg)
        raise RuntimeError(f"dgb200 error {rc}: {msg}")


class RasterDesc(ctypes.Structure):
    _fields_ = [("nx", c_int), ("ny", c_int), ("max_nodes", c_int), ("block_nodes", c_int * MAX_BLOCKS),
                ("pixel_block", c_void_p), ("pixel_element", c_void_p), ("pixel_weights", c_void_p),
                ("body_mask", c_void_p), ("grad_mask", c_void_p), ("luts", c_void_p),
                ("background", ctypes.c_uint8 * 4), ("dx", ctypes.c_double), ("dy", ctypes.c_double)]


def dptr(a, ctype=ctypes.c_double):
    """Pointer to a C-contiguous numpy array (the caller keeps the array alive)."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def affine_test(J, tol):
    """(affine uint8[E], mean[E][9]) of per-point inverse Jacobians J (E, Nq, 9) on host threads
    (``dgb_affine_test``)."""
    J = as_f64(J)
    E = J.shape[0]
    affine = np.empty(E, np.uint8)
    mean = np.empty((E, 9))
    check(lib().dgb_affine_test(dptr(J), E, J.shape[1], float(tol), dptr(affine, ctypes.c_uint8), dptr(mean)))
    return affine, mean


def pair_faces(keys, visit):
    """(owner rows, neighbour rows, -1 at the boundary) of the faces of one face type, in the
    reference's face order, from the visits' sorted corner keys (n, k) and visiting order (n,)
    (``dgb_pair_faces``, host threads)."""
    keys = np.ascontiguousarray(keys, np.int64)
    visit = np.ascontiguousarray(visit, np.int64)
    n, k = keys.shape
    owner = np.empty(max(n, 1), np.int64)
    neighbor = np.empty(max(n, 1), np.int64)
    count = ctypes.c_int64(0)
    check(lib().dgb_pair_faces(dptr(keys, ctypes.c_int64), k, n, dptr(visit, ctypes.c_int64),
                               dptr(owner, ctypes.c_int64), dptr(neighbor, ctypes.c_int64), ctypes.byref(count)))
    return owner[:count.value], neighbor[:count.value]


def msh_nodes(body, count, version):
    """(node ids (n,), coordinates (n, 3)) of a Gmsh ASCII $Nodes section body (bytes after the
    "$Nodes" line; for MSH 2.2 after the count line): ``dgb_msh2_nodes`` / ``dgb_msh4_nodes``."""
    ids = np.empty(max(count, 1), np.int64)
    xyz = np.empty((max(count, 1), 3))
    fn = lib().dgb_msh2_nodes if version == 2 else lib().dgb_msh4_nodes
    check(fn(body, len(body), count, dptr(ids, ctypes.c_int64), dptr(xyz)))
    return ids[:count], xyz[:count]


def msh_elements(body, count, version, cap):
    """Element records of a Gmsh ASCII $Elements section body, at most cap node ids in all: MSH 2.2
    (type, physical tag, offsets, node ids); MSH 4.1 (type, entity dimension, entity tag, offsets,
    node ids) (``dgb_msh2_elements`` / ``dgb_msh4_elements``)."""
    n = max(count, 1)
    cap = max(int(cap), 1)
    t, a, b = (np.empty(n, np.int32) for _ in range(3))
    offsets = np.empty(n + 1, np.int64)
    nodes = np.empty(cap, np.int64)
    P32, P64 = ctypes.c_int32, ctypes.c_int64
    if version == 2:
        check(lib().dgb_msh2_elements(body, len(body), count, dptr(t, P32), dptr(a, P32), dptr(offsets, P64),
                                      dptr(nodes, P64), cap))
        return t[:count], a[:count], offsets[:count + 1], nodes[:offsets[count]]
    check(lib().dgb_msh4_elements(body, len(body), count, dptr(t, P32), dptr(a, P32), dptr(b, P32),
                                  dptr(offsets, P64), dptr(nodes, P64), cap))
    return t[:count], a[:count], b[:count], offsets[:count + 1], nodes[:offsets[count]]


def as_f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def as_i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def map_metrics(nodes, grad, index=None, weights=None, tangents=None, orientation=None,
                outputs=("det", "inv_jacobian")):
    """Geometry metrics on the host cores (``dgb_map_metrics``): element i of the result maps
    by nodes[index[i]] (all of ``nodes`` when ``index`` is None) at the points of ``grad``
    (Q, n, 3).  ``outputs`` names the arrays to return, in that order, from jacobian (count, Q,
    3, 3), det (count, Q), inv_jacobian (count, Q, 3, 3), wdet (count, Q), normals (count, Q, 3)
    and area_weights (count, Q)."""
    nodes = as_f64(nodes)
    grad = as_f64(grad)
    idx = None if index is None else as_i32(index)
    if idx is not None and len(idx) and (idx.min() < 0 or idx.max() >= len(nodes)):
        raise ValueError(f"element index out of range for {len(nodes)} node sets")
    count = len(nodes) if idx is None else len(idx)
    Q, n = grad.shape[0], grad.shape[1]
    if nodes.shape[1:] != (n, 3):
        raise ValueError(f"nodes have shape {nodes.shape}; the geometry basis has {n} nodes")
    shapes = dict(jacobian=(count, Q, 3, 3), det=(count, Q), inv_jacobian=(count, Q, 3, 3), wdet=(count, Q),
                  normals=(count, Q, 3), area_weights=(count, Q))
    out = {k: np.empty(shapes[k]) for k in outputs}
    keep = [None if a is None else as_f64(a) for a in (weights, tangents, orientation)]
    args = [None if a is None else dptr(a) for a in keep]
    check(lib().dgb_map_metrics(dptr(nodes), None if idx is None else dptr(idx, ctypes.c_int32), count, n,
                                dptr(grad), Q, *args,
                                *[dptr(out[k]) if k in out else None for k in shapes]))
    return tuple(out[k] for k in outputs)


def subcell_face_metrics(vertices, centers, faces, owners, neighbors=None):
    """Subcell face metrics on the host cores (``dgb_subcell_face_metrics``): vertices (E, V, 3),
    centers (E, S, 3), faces a list of 3- or 4-vertex id sequences; returns unit normals (E, F, 3),
    areas (E, F) and face centres (E, F, 3)."""
    vertices, centers = as_f64(vertices), as_f64(centers)
    E, V, _ = vertices.shape
    F = len(faces)
    table = np.zeros((max(F, 1), 4), np.int32)
    sizes = np.zeros(max(F, 1), np.int32)
    for f, face in enumerate(faces):
        table[f, :len(face)] = face
        sizes[f] = len(face)
    own = as_i32(owners)
    nbr = None if neighbors is None else as_i32(neighbors)
    normals, areas, fc = np.empty((E, F, 3)), np.empty((E, F)), np.empty((E, F, 3))
    check(lib().dgb_subcell_face_metrics(dptr(vertices), E, V, dptr(table, ctypes.c_int32), dptr(sizes, ctypes.c_int32),
                                         F, dptr(centers), centers.shape[1], dptr(own, ctypes.c_int32),
                                         None if nbr is None else dptr(nbr, ctypes.c_int32), dptr(normals), dptr(areas),
                                         dptr(fc)))
    return normals, areas, fc
