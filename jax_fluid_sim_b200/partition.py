"""Element partition of one mesh over several GPUs (one process per GPU) with a one-layer
element halo, and the SSP-RK3 step that exchanges it.

The reference runs on one device and has no counterpart.  The DG residual of an element depends
on its own state and on its face neighbours' states only (the traces at shared faces, and for
BR2 the neighbour's local lift, hybrid/spatial.py:137-234, hybrid/navier_stokes.py:138-336).
So each rank holds:
  - its owned elements (recursive coordinate bisection of the element centroids), and
  - one layer of ghost elements: the other ranks' elements that share a face with an owned one;
and builds an ordinary single-GPU plan over owned + ghost elements.  Before every residual the
ghost states are refreshed from their owners (one exchange per RK stage); the residuals of the
owned elements are then exactly those of the whole mesh, and the ghosts' own residuals (whose
outer faces are cut) are never used.  Faces of ghosts that lead out of the rank's elements carry
the physical tag ``partition``, which no boundary role names, so their ghost is the interior
trace.

What needs more than the owned elements' own data is reduced over ranks: the stable dt (min),
admissibility (AND of the valid flags, min of rho and p).  The positivity limiter is element-local.
The MOOD recompute is not partitioned (its detector flags of ghosts would need a second exchange
per stage), nor are periodic or curved meshes.

Transport is ``torch.distributed`` point-to-point (batched isend/irecv): NCCL over NVLink between
GPUs, gloo on the CPU.  Remote states land in this rank's own buffers before any kernel reads
them (no kernel reads a peer's memory).
"""

import numpy as np

from . import meshgen
from .meshgen import MeshSource

PARTITION_TAG_NAME = "partition"
BLOCK_ORDER = ("hexahedron", "wedge", "tetra")


def rcb(points, parts):
    """Recursive coordinate bisection: part id in [0, parts) of each point.  Each cut splits
    along the widest extent of the points it divides, at the count proportional to the parts
    on each side (stable sort, so ties split deterministically)."""
    points = np.asarray(points, np.float64)
    out = np.zeros(len(points), np.int32)

    def split(ids, first, count):
        if count == 1 or len(ids) == 0:
            out[ids] = first
            return
        left = count // 2
        axis = int(np.argmax(np.ptp(points[ids], axis=0)))
        order = ids[np.argsort(points[ids, axis], kind="stable")]
        cut = int(round(len(ids) * left / count))
        split(order[:cut], first, left)
        split(order[cut:], first + left, count - left)

    split(np.arange(len(points)), 0, int(parts))
    return out


class ElementPartition:
    """Parts of a HybridMesh's elements (global element id = position in block order)."""

    def __init__(self, mesh, parts, part_of=None):
        if mesh.source.periodic_map is not None:
            raise NotImplementedError("periodic meshes are not partitioned")
        if any(b.geometry_connectivity is not None for b in mesh.element_blocks):
            raise NotImplementedError("curved (second-order geometry) meshes are not partitioned")
        self.mesh = mesh
        self.parts = int(parts)
        sizes = [len(b.connectivity) for b in mesh.element_blocks]
        self.offsets = np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)
        centers = np.concatenate([b.centers for b in mesh.element_blocks])
        self.part = rcb(centers, parts) if part_of is None else np.asarray(part_of, np.int32)
        if len(self.part) != self.offsets[-1]:
            raise ValueError("one part per element is needed")

    def global_id(self, block, local):
        return self.offsets[block] + np.asarray(local, np.int64)


class LocalDomain:
    """One rank's owned and ghost elements and its mesh source.

    Local element order per block: owned elements by global id, then ghosts by global id.
    ``source`` is a MeshSource of those elements (points compacted, boundary faces tagged as in
    the whole mesh, cut faces of ghosts tagged ``partition``).  ``send[peer][etype]`` lists the
    local indices of owned elements that ``peer`` holds as ghosts, ``recv[peer][etype]`` the local
    indices of this rank's ghosts owned by ``peer``, both in global-id order, so that the k-th
    sent state is the k-th received one."""

    def __init__(self, partition: ElementPartition, rank):
        mesh, part = partition.mesh, partition.part
        self.rank, self.parts = int(rank), partition.parts
        ghosts = set()
        for fb in mesh.face_blocks.values():
            inner = np.flatnonzero(fb.neighbor_block >= 0)
            go = partition.offsets[fb.owner_block[inner]] + fb.owner_local[inner]
            gn = partition.offsets[fb.neighbor_block[inner]] + fb.neighbor_local[inner]
            po, pn = part[go], part[gn]
            ghosts.update(gn[(po == rank) & (pn != rank)].tolist())
            ghosts.update(go[(pn == rank) & (po != rank)].tolist())
        self.blocks = []          # (etype, global ids in local order, number owned)
        for b, blk in enumerate(mesh.element_blocks):
            ids = np.arange(partition.offsets[b], partition.offsets[b + 1])
            owned = ids[part[ids] == rank]
            gh = np.asarray(sorted(g for g in ghosts if partition.offsets[b] <= g < partition.offsets[b + 1]),
                            np.int64)
            if len(owned) + len(gh):          # a block with no local element is left out
                self.blocks.append((blk.element_type, np.concatenate([owned, gh]).astype(np.int64), len(owned)))
        self.owned = {etype: n for etype, _, n in self.blocks}
        self.global_ids = {etype: g for etype, g, _ in self.blocks}
        self.source = self._source(partition)
        # exchange lists
        local_index = {}
        for etype, g, _ in self.blocks:
            local_index.update({int(x): (etype, i) for i, x in enumerate(g)})
        self.send = {p: {e: [] for e, _, _ in self.blocks} for p in range(self.parts) if p != rank}
        self.recv = {p: {e: [] for e, _, _ in self.blocks} for p in range(self.parts) if p != rank}
        for etype, g, n in self.blocks:
            for i in range(n, len(g)):                       # ghosts: received from their owner
                self.recv[int(part[g[i]])][etype].append(i)
        # an owned element is sent to every rank that holds it as a ghost: the ranks of its
        # face neighbours (other than this one)
        for fb in mesh.face_blocks.values():
            inner = np.flatnonzero(fb.neighbor_block >= 0)
            go = partition.offsets[fb.owner_block[inner]] + fb.owner_local[inner]
            gn = partition.offsets[fb.neighbor_block[inner]] + fb.neighbor_local[inner]
            for a, b in ((go, gn), (gn, go)):
                mask = (part[a] == rank) & (part[b] != rank)
                for x, peer in zip(a[mask].tolist(), part[b[mask]].tolist()):
                    etype, i = local_index[x]
                    self.send[peer][etype].append(i)
        for peer in self.send:
            for etype, g, _ in self.blocks:
                idx = sorted(set(self.send[peer][etype]), key=lambda i: g[i])
                self.send[peer][etype] = np.asarray(idx, np.int64)
                self.recv[peer][etype] = np.asarray(sorted(self.recv[peer][etype], key=lambda i: g[i]), np.int64)

    def _source(self, partition):
        mesh = partition.mesh
        cells, used = [], []
        index = {blk.element_type: b for b, blk in enumerate(mesh.element_blocks)}
        for etype, g, _ in self.blocks:
            b = index[etype]
            conn = mesh.element_blocks[b].connectivity[g - partition.offsets[b]]
            cells.append((etype, conn))
            used.append(conn.ravel())
        pts = np.unique(np.concatenate(used)) if used else np.zeros(0, np.int64)
        remap = np.full(len(mesh.points), -1, np.int64)
        remap[pts] = np.arange(len(pts))
        # boundary tags of the whole mesh by sorted node key
        tag_of = {}
        for fb in mesh.face_blocks.values():
            for nodes, t in zip(fb.nodes[fb.neighbor_block < 0], fb.boundary_tags[fb.neighbor_block < 0]):
                tag_of[tuple(sorted(int(v) for v in nodes))] = int(t)
        field = dict(mesh.source.field_data)
        cut_tag = max([v[0] for v in field.values()] + [0]) + 1
        field[PARTITION_TAG_NAME] = (cut_tag, 2)
        seen = {}
        for etype, conn in cells:
            for cell in conn:
                for loc in meshgen.FACES[etype]:
                    nodes = tuple(int(cell[i]) for i in loc)
                    key = tuple(sorted(nodes))
                    seen[key] = (seen[key][0] + 1, nodes) if key in seen else (1, nodes)
        tris, quads, ttag, qtag = [], [], [], []
        for key, (count, nodes) in seen.items():
            if count != 1:
                continue
            t = tag_of.get(key, cut_tag)
            (tris if len(nodes) == 3 else quads).append([remap[v] for v in nodes])
            (ttag if len(nodes) == 3 else qtag).append(t)
        volume_tag = field.get("fluid", (0, 3))[0]
        out_cells = [(etype, remap[conn].astype(np.int32)) for etype, conn in cells if len(conn)]
        phys = [np.full(len(conn), volume_tag, np.int32) for etype, conn in cells if len(conn)]
        if tris:
            out_cells.append(("triangle", np.asarray(tris, np.int32)))
            phys.append(np.asarray(ttag, np.int32))
        if quads:
            out_cells.append(("quad", np.asarray(quads, np.int32)))
            phys.append(np.asarray(qtag, np.int32))
        return MeshSource(mesh.points[pts], out_cells, phys, field, None)

    def owned_view(self, states):
        """The owned elements' rows of local ``states``."""
        return {etype: states[etype][:n] for etype, n in self.owned.items() if etype in states and n > 0}


class HaloExchange:
    """Refreshes the ghost rows of local states from their owners (torch.distributed
    point-to-point, one batched round per call; every rank calls it at the same points)."""

    def __init__(self, domain: LocalDomain, group=None):
        self.domain = domain
        self.group = group

    def __call__(self, states):
        import torch
        import torch.distributed as dist
        ops, inbox = [], []
        for peer in sorted(self.domain.send):
            for etype in BLOCK_ORDER:
                if etype not in states:
                    continue
                s_idx, r_idx = self.domain.send[peer][etype], self.domain.recv[peer][etype]
                U = states[etype]
                if len(s_idx):
                    buf = U[torch.as_tensor(s_idx, device=U.device)].contiguous()
                    ops.append(dist.P2POp(dist.isend, buf, peer, self.group))
                    inbox.append((None, buf))
                if len(r_idx):
                    buf = torch.empty((len(r_idx),) + tuple(U.shape[1:]), dtype=U.dtype, device=U.device)
                    ops.append(dist.P2POp(dist.irecv, buf, peer, self.group))
                    inbox.append(((etype, r_idx), buf))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for target, buf in inbox:
            if target is not None:
                etype, r_idx = target
                states[etype][torch.as_tensor(r_idx, device=buf.device)] = buf
        return states


def _allreduce(value, op, device):
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


class PartitionedSSPRK3:
    """Checked SSP-RK3 step (hybrid/time_integration.py:404-583, non-MOOD branch) of one rank's
    local states: before each stage's residual the ghosts are refreshed; the stage update and the
    element-local limiter run on all local rows; admissibility is taken over the owned rows and
    reduced over ranks.  ``rhs(states)`` and ``limiter(states)`` (optional) act on local state
    dicts (the GPU operator of the local plan, or any function with that contract);
    ``admissibility(states)`` returns (valid, rho_min, p_min) of the states it is given."""

    STAGES = ((0.0, 1.0), (0.75, 0.25), (1.0 / 3.0, 2.0 / 3.0))

    def __init__(self, domain, exchange, rhs, admissibility, limiter=None, device="cpu"):
        self.domain, self.exchange, self.rhs = domain, exchange, rhs
        self.admissibility, self.limiter, self.device = admissibility, limiter, device

    def stable_dt(self, local_dt):
        """The smallest of every rank's local stable dt."""
        import torch.distributed as dist
        return _allreduce(local_dt, dist.ReduceOp.MIN, self.device)

    def checked_step(self, states, dt):
        import torch.distributed as dist
        base = {k: v for k, v in states.items()}
        self.exchange(base)
        cur, valid, rmin, pmin = base, True, np.inf, np.inf
        for s, (alpha, beta) in enumerate(self.STAGES):
            if s > 0:
                self.exchange(cur)
            R = self.rhs(cur)
            new = {k: alpha * base[k] + beta * (cur[k] + dt * R[k]) for k in cur}
            if self.limiter is not None:
                new = self.limiter(new)
            v, r, p = self.admissibility(self.domain.owned_view(new))
            valid, rmin, pmin = valid and bool(v), min(rmin, float(r)), min(pmin, float(p))
            cur = new
        valid = _allreduce(1.0 if valid else 0.0, dist.ReduceOp.MIN, self.device) > 0.5
        rmin = _allreduce(rmin, dist.ReduceOp.MIN, self.device)
        pmin = _allreduce(pmin, dist.ReduceOp.MIN, self.device)
        self.exchange(cur)
        return cur, valid, rmin, pmin
