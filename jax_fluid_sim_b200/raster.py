"""Midplane rasteriser into a headless RGBA buffer (reference: ``GPUMidplaneRasterizer``,
hybrid/gui/gpu_rasterizer.py:18-344).

The reference cuts the elements' visualisation subcells with the plane z = plane_z, averages
the cut points and samples the pixel grid by 2-D Delaunay barycentric interpolation.  Here each
pixel is located in its element on the host once (candidate elements by centroid distance, the
element map inverted by Newton's method), and the device evaluates the element's nodal
primitives with the solution basis at that point: the same field the DG solution holds there,
with no triangulation of the cut.  Framing, body and gradient masks, display modes, default
limits and the shock palette follow the reference (hybrid/output.py:10-28 for the palette);
the temperature palette is this module's own black-red-yellow-white ramp (the reference uses a
plotting library's "inferno" table).  There is no window: ``render`` returns the (ny, nx, 4)
uint8 image as a CUDA tensor.
"""

import ctypes

import numpy as np
import torch

from . import _native as N

SHOCK_STOPS = ((0.00, "#01051f"), (0.18, "#031b5c"), (0.38, "#054e99"), (0.55, "#00a3d9"),
               (0.70, "#1ec98b"), (0.82, "#e0d825"), (0.92, "#ff6a14"), (1.00, "#ff1a10"))
HEAT_STOPS = ((0.0, "#000004"), (0.35, "#8a1c1c"), (0.7, "#f2a01b"), (1.0, "#fcffa4"))
BACKGROUND = (1, 5, 31, 255)
DEFAULT_LIMITS = {0: (0.0, 1.0), 1: (0.5, 5.0), 2: (0.5, 10.0), 3: (0.0, 6.0), 4: (250.0, 3800.0)}


def palette(stops, n=256):
    """(n, 4) uint8 table: piecewise-linear RGB through the colour stops at k / (n - 1), opaque."""
    pos = np.asarray([s[0] for s in stops])
    rgb = np.asarray([[int(c[i:i + 2], 16) / 255.0 for i in (1, 3, 5)] for _, c in stops])
    x = np.linspace(0.0, 1.0, n)
    out = np.ones((n, 4))
    for ch in range(3):
        out[:, ch] = np.interp(x, pos, rgb[:, ch])
    return (out * 255.0).astype(np.uint8)


def _inside(etype, xi, tol=1.0e-9):
    if etype == "hexahedron":
        return np.all((xi >= -tol) & (xi <= 1.0 + tol), axis=-1)
    if etype == "wedge":
        return ((xi[..., 0] >= -tol) & (xi[..., 1] >= -tol) & (xi[..., 0] + xi[..., 1] <= 1.0 + tol)
                & (xi[..., 2] >= -tol) & (xi[..., 2] <= 1.0 + tol))
    return np.all(xi >= -tol, axis=-1) & (xi.sum(axis=-1) <= 1.0 + tol)


class GPUMidplaneRasterizer:
    def __init__(self, operator, resolution=(800, 450), plane_z=0.0, sphere_radius=0.5, sphere_center=(0.0, 0.0),
                 candidates=12):
        from scipy.spatial import cKDTree
        self.operator = operator
        self.solver = operator.solver
        self.nx, self.ny = resolution
        self.plane_z = float(plane_z)
        self.sphere_radius = float(sphere_radius)
        self.sphere_center = tuple(sphere_center)
        mesh, plan = operator.mesh, operator.plan
        # elements that cross the plane, and the plane's cut of their corner edges (framing)
        cut_xy, crossing = [], []
        for b, block in enumerate(mesh.element_blocks):
            geo, xyz = mesh.geometry(block)
            z = mesh.points[block.connectivity][..., 2]
            hit = np.flatnonzero((z.min(axis=1) <= self.plane_z + 1e-10) & (z.max(axis=1) >= self.plane_z - 1e-10))
            crossing.append(hit)
            c = mesh.points[block.connectivity[hit]]
            cut_xy.append(c[..., :2].reshape(-1, 2))
        allxy = np.concatenate(cut_xy) if cut_xy else np.zeros((1, 2))
        raw_xmin, raw_ymin = allxy.min(axis=0)
        raw_xmax, raw_ymax = allxy.max(axis=0)
        axisymmetric = raw_ymin >= -1.0e-3
        if axisymmetric:                            # gpu_rasterizer.py:117-130
            aspect = self.nx / self.ny
            half_height = 1.35
            total_width = 2.0 * half_height * aspect
            self.xmin = 0.55 - total_width * 0.42
            self.xmax = self.xmin + total_width
            self.ymin, self.ymax = -half_height, half_height
        else:
            self.xmin, self.xmax, self.ymin, self.ymax = raw_xmin, raw_xmax, raw_ymin, raw_ymax
        self.extent = (self.xmin, self.xmax, self.ymin, self.ymax)
        gx = np.linspace(self.xmin, self.xmax, self.nx)
        gy = np.linspace(self.ymax, self.ymin, self.ny)          # row 0 at the top
        GX, GY = np.meshgrid(gx, gy)
        pts = np.column_stack([GX.ravel(), np.abs(GY.ravel()) if axisymmetric else GY.ravel(),
                               np.full(GX.size, self.plane_z)])
        npix = len(pts)
        max_np = max(bp.Np for bp in plan.blocks)
        pix_block = np.full(npix, -1, np.int32)
        pix_elem = np.zeros(npix, np.int32)
        pix_w = np.zeros((npix, max_np), np.float32)
        for b, (block, bp) in enumerate(zip(mesh.element_blocks, plan.blocks)):
            hit = crossing[b]
            if not len(hit):
                continue
            geo, xyz_all = mesh.geometry(block)
            xyz = xyz_all[hit]
            tree = cKDTree(xyz.mean(axis=1))
            todo = np.flatnonzero(pix_block < 0)
            k = min(candidates, len(hit))
            _, cand = tree.query(pts[todo], k=k)
            cand = cand.reshape(len(todo), k)
            for c in range(k):
                todo_c = todo[pix_block[todo] < 0]
                if not len(todo_c):
                    break
                sel = np.searchsorted(todo, todo_c)
                elems = cand[sel, c]
                X = xyz[elems]                                        # (m, ng, 3)
                xi = np.broadcast_to(geo.nodes.mean(axis=0), (len(elems), 3)).copy()
                for _ in range(12):
                    Nb = geo.basis(xi)
                    G = geo.basis_gradients(xi)
                    x = np.einsum("mk,mkd->md", Nb, X)
                    J = np.einsum("mkd,mkr->mdr", X, G)
                    xi = xi - np.einsum("mrd,md->mr", np.linalg.inv(J), x - pts[todo_c])
                ok = _inside(block.element_type, xi)
                found = todo_c[ok]
                pix_block[found] = b
                pix_elem[found] = hit[elems[ok]]
                pix_w[found, :bp.Np] = bp.ref.basis(xi[ok]).astype(np.float32)
        self.dx, self.dy = abs(float(gx[1] - gx[0])), abs(float(gy[1] - gy[0]))
        r_sq = (GX.ravel() - self.sphere_center[0]) ** 2 + (GY.ravel() - self.sphere_center[1]) ** 2
        self.sphere_mask = (r_sq < (self.sphere_radius + 1.0e-4) ** 2).reshape(self.ny, self.nx)
        pad = 1.5 * max(self.dx, self.dy)
        self.grad_mask = (r_sq < (self.sphere_radius + pad) ** 2).reshape(self.ny, self.nx)
        pix_block[self.sphere_mask.ravel()] = -1
        self.coverage = float(np.mean(pix_block >= 0))
        self.pixel_points = pts
        self.pixel_block, self.pixel_element, self.pixel_weights = pix_block, pix_elem, pix_w
        self._max_np = max_np
        self._desc = None

    def _upload(self):
        plan = self.operator.plan
        pix_block, pix_elem, pix_w, max_np = self.pixel_block, self.pixel_element, self.pixel_weights, self._max_np
        dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")
        self._buffers = dict(block=dev(pix_block), elem=dev(pix_elem), w=dev(pix_w),
                             body=dev(self.sphere_mask.astype(np.uint8)), grad=dev(self.grad_mask.astype(np.uint8)),
                             luts=dev(np.stack([palette(SHOCK_STOPS), palette(HEAT_STOPS)])))
        d = N.RasterDesc()
        d.nx, d.ny, d.max_nodes = self.nx, self.ny, max_np
        for b, bp in enumerate(plan.blocks):
            d.block_nodes[b] = bp.Np
        d.pixel_block = self._buffers["block"].data_ptr()
        d.pixel_element = self._buffers["elem"].data_ptr()
        d.pixel_weights = self._buffers["w"].data_ptr()
        d.body_mask = self._buffers["body"].data_ptr()
        d.grad_mask = self._buffers["grad"].data_ptr()
        d.luts = self._buffers["luts"].data_ptr()
        for k in range(4):
            d.background[k] = BACKGROUND[k]
        d.dx, d.dy = self.dx, self.dy
        self._desc = d
        self._grid = torch.empty((self.ny, self.nx, 5), dtype=torch.float64, device="cuda")
        self._rgba = torch.empty((self.ny, self.nx, 4), dtype=torch.uint8, device="cuda")

    def render(self, states, mode=0, vmin=None, vmax=None):
        """gpu_rasterizer.py:290-344: mode 0 schlieren, 1 density, 2 pressure, 3 Mach, 4 temperature;
        returns (rgba (ny, nx, 4) uint8 CUDA tensor, vmin, vmax)."""
        if vmin is None or vmax is None:
            vmin, vmax = DEFAULT_LIMITS[int(mode) if int(mode) in DEFAULT_LIMITS else 4]
        if self._desc is None:
            self._upload()
        U = self.operator.to_device(states)
        st = self.operator.native.state(self.operator._blocks(U))
        N.check(N.lib().dgb_raster_render(ctypes.byref(self._desc), ctypes.byref(st),
                                          self.solver.layout.number_of_variables, self.solver.gamma, int(mode),
                                          float(vmin), float(vmax), ctypes.c_void_p(self._grid.data_ptr()),
                                          ctypes.c_void_p(self._rgba.data_ptr()),
                                          ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        return self._rgba, float(vmin), float(vmax)
