"""Element partition with a one-layer ghost halo (jax_fluid_sim_b200.partition), on the CPU.

Single process: the recursive coordinate bisection is balanced, every element is owned once, the
exchange lists of each pair of ranks match, and the local mesh builds.  Two gloo ranks
(127.0.0.1): each rank evaluates the residual of its owned + ghost elements on its own local
mesh, refreshed by the halo exchange, and takes one checked SSP-RK3 step with the positivity
limiter; the owned elements' residuals and stepped states equal the whole mesh's to 1e-12 of
each field's largest magnitude (float64, the same operator applied to the same traces).  The
residuals come from the oracle (the kernels need a GPU); the partition, the exchange and the
step driver under test are the product's."""

import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from jax_fluid_sim_b200 import HybridMesh, meshgen
from jax_fluid_sim_b200.partition import ElementPartition, LocalDomain, rcb

FARFIELD = [1.0, 0.6, 0.1, 0.0, 1.0]


def _mesh(kind="box"):
    """A jittered hexahedron box with far-field, wall and no-slip planes, or the golden smoke
    mesh (hexahedra, prisms and tetrahedra)."""
    if kind == "box":
        src = meshgen.box_hex((5, 3, 3), hi=(1.5, 1.0, 1.0), jitter=0.1, seed=3)
    else:
        from .conftest import load_golden
        src = load_golden("smoke_p2")["source"]
    return src, HybridMesh(src)


def _oracle(source, degree=2, mu=0.01):
    from oracle.dg import Operator, PositivityLimiter, TimeIntegrator
    from oracle.mesh import Mesh, MeshSource
    from oracle.physics import FarfieldWallBoundary, Gas
    mesh = Mesh(MeshSource(source.points, source.cells, source.physical, source.field_data, None))
    gas = Gas(dynamic_viscosity=mu)
    op = Operator(mesh, gas, degree)
    bc = FarfieldWallBoundary(gas, mesh.physical_names, FARFIELD, wall_temperature=1.2)
    integ = TimeIntegrator(op, cfl=0.3, limiter=PositivityLimiter(op))
    return op, bc, integ


def _state(op):
    from oracle.elements import RefElement
    out = {}
    for b in op.mesh.element_blocks:
        nodes = RefElement(b.element_type, op.degree).nodes
        x = np.einsum("qi,eid->eqd", RefElement(b.element_type, 1).basis(nodes), op.mesh.points[b.connectivity])
        W = np.stack([1 + 0.1 * np.sin(3 * x[..., 0]), 0.5 + 0.1 * np.cos(x[..., 1]), 0.1 * np.cos(2 * x[..., 1]),
                      0.05 * x[..., 2], 1 + 0.05 * np.cos(x[..., 2])], -1)
        out[b.element_type] = op.gas.to_conserved(W)
    return out


@pytest.mark.parametrize("kind", ["box", "smoke"])
def test_rcb_and_local_domains(kind):
    src, mesh = _mesh(kind)
    part = ElementPartition(mesh, 3)
    counts = np.bincount(part.part, minlength=3)
    assert counts.sum() == part.offsets[-1] and counts.max() - counts.min() <= 1
    doms = [LocalDomain(part, r) for r in range(3)]
    owned = np.concatenate([d.global_ids[e][:d.owned[e]] for d in doms for e in d.owned])
    assert np.array_equal(np.sort(owned), np.arange(part.offsets[-1]))
    for a in doms:
        for b in doms:
            if a is b:
                continue
            for e in a.owned:
                sa = a.send[b.rank][e]
                if e not in b.owned:
                    assert len(sa) == 0
                    continue
                rb = b.recv[a.rank][e]
                assert np.array_equal(a.global_ids[e][sa], b.global_ids[e][rb])
        local = HybridMesh(a.source)          # builds and validates
        assert [blk.element_type for blk in local.element_blocks] == [e for e, _, _ in a.blocks]
    assert rcb(np.zeros((5, 3)), 2).tolist().count(0) in (2, 3)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, kind, out):
    import os
    import torch.distributed as dist
    from oracle.dg import PositivityLimiter
    from jax_fluid_sim_b200.partition import HaloExchange, PartitionedSSPRK3
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        src, mesh = _mesh(kind)
        gop, gbc, ginteg = _oracle(src)
        U = _state(gop)
        dt = ginteg.stable_dt(U)
        ref_rhs = gop.rhs(U, gbc)
        ref_step, ref_valid, ref_rmin, ref_pmin = ginteg.checked_step(U, dt, gbc)
        part = ElementPartition(mesh, world)
        dom = LocalDomain(part, rank)
        lop, lbc, linteg = _oracle(dom.source)
        offs = {b.element_type: part.offsets[k] for k, b in enumerate(mesh.element_blocks)}
        # local states: owned rows from the global state, ghost rows left at zero for the exchange
        local = {}
        for etype, g, n in dom.blocks:
            arr = np.zeros((len(g),) + U[etype].shape[1:])
            arr[:n] = U[etype][g[:n] - offs[etype]]
            local[etype] = torch.from_numpy(arr)
        ex = HaloExchange(dom)
        ex(local)
        to_np = lambda st: {k: v.numpy() for k, v in st.items()}
        to_t = lambda st: {k: torch.from_numpy(np.ascontiguousarray(v)) for k, v in st.items()}
        rhs = lop.rhs(to_np(local), lbc)
        errs = []
        for etype, g, n in dom.blocks:
            if n == 0:
                continue
            ref = ref_rhs[etype]
            errs.append(np.max(np.abs(rhs[etype][:n] - ref[g[:n] - offs[etype]])) / np.max(np.abs(ref)))
        stepper = PartitionedSSPRK3(dom, ex, rhs=lambda st: to_t(lop.rhs(to_np(st), lbc)),
                                    admissibility=lambda st: linteg.admissibility(to_np(st)),
                                    limiter=lambda st: to_t(PositivityLimiter(lop)(to_np(st))))
        assert abs(stepper.stable_dt(linteg.stable_dt(to_np(local))) - dt) <= 1e-15 * dt
        new, valid, rmin, pmin = stepper.checked_step(local, dt)
        serr = []
        for etype, g, n in dom.blocks:
            if n == 0:
                continue
            ref = ref_step[etype]
            serr.append(np.max(np.abs(new[etype][:n].numpy() - ref[g[:n] - offs[etype]])) / np.max(np.abs(ref)))
        out[rank] = (max(errs), max(serr), valid == ref_valid, abs(rmin - ref_rmin) <= 1e-14 * abs(ref_rmin),
                     abs(pmin - ref_pmin) <= 1e-14 * abs(ref_pmin), sum(n for _, _, n in dom.blocks))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("kind", ["box", "smoke"])
def test_two_ranks_match_whole_mesh(kind):
    world = 2
    with mp.Manager() as manager:
        out = manager.dict()
        mp.spawn(_rank_main, args=(world, _free_port(), kind, out), nprocs=world, join=True)
        res = dict(out)
    assert sorted(res) == [0, 1]
    for rank, (rhs_err, step_err, valid_ok, rmin_ok, pmin_ok, owned) in res.items():
        assert rhs_err <= 1e-12, (rank, rhs_err)
        assert step_err <= 1e-12, (rank, step_err)
        assert valid_ok and rmin_ok and pmin_ok
        assert owned > 0
