"""Midplane rasteriser: pixel location on the host (CPU) and the rendered image on the GPU
(reference test: tests/test_gpu_rasterizer.py:24-60 -- shape, dtype, the body's background
pixel, every display mode; here also the interpolated field itself)."""

import numpy as np
import pytest

from jax_fluid_sim_b200 import meshgen
from jax_fluid_sim_b200.raster import BACKGROUND, GPUMidplaneRasterizer, SHOCK_STOPS, palette


@pytest.fixture(scope="module")
def raster_cpu():
    """Operator-free construction needs a plan only: build one through the public classes."""
    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200.plan import Plan

    class _Op:
        pass
    src = meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))
    mesh = jfs.HybridMesh(src)
    op = _Op()
    op.mesh, op.plan = mesh, Plan(mesh, 2)
    op.solver = type("S", (), {"gamma": 1.4})()
    return GPUMidplaneRasterizer(op, resolution=(160, 90))


def test_palette_ends_and_shape():
    lut = palette(SHOCK_STOPS)
    assert lut.shape == (256, 4) and lut.dtype == np.uint8
    np.testing.assert_array_equal(lut[0], [1, 5, 31, 255])
    np.testing.assert_array_equal(lut[-1], [255, 26, 16, 255])


def test_pixels_located_in_their_elements(raster_cpu):
    r = raster_cpu
    assert r.coverage > 0.9
    assert r.sphere_mask.any() and r.grad_mask.sum() >= r.sphere_mask.sum()
    mesh = r.operator.mesh
    for b, block in enumerate(mesh.element_blocks):
        sel = np.flatnonzero(r.pixel_block == b)[::37]
        geo, xyz = mesh.geometry(block)
        bp = r.operator.plan.blocks[b]
        # the solution basis reproduces linear functions: sum_i w_i x_i = the pixel point
        x_nodes = bp.node_xyz[r.pixel_element[sel]]
        x = np.einsum("pi,pid->pd", r.pixel_weights[sel, :bp.Np].astype(np.float64), x_nodes)
        np.testing.assert_allclose(x, r.pixel_points[sel], atol=2e-6)


@pytest.mark.gpu
def test_render_modes_and_field():
    import torch
    import jax_fluid_sim_b200 as jfs
    src = meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=2, dynamic_viscosity=1e-3)
    op = jfs.HybridNavierStokesOperator(solver)
    r = GPUMidplaneRasterizer(op, resolution=(640, 360))
    states = solver.uniform_state_blocks(1.2, [1500.0, 0.0, 0.0], 101325.0)
    for mode in range(5):
        rgba, vmin, vmax = r.render(states, mode=mode)
        assert rgba.shape == (360, 640, 4) and rgba.dtype == torch.uint8
    cx = int(640 * (0.0 - r.xmin) / (r.xmax - r.xmin))
    cy = int(360 * (0.0 - r.ymin) / (r.ymax - r.ymin))
    np.testing.assert_array_equal(rgba[cy, cx].cpu().numpy(), BACKGROUND)
    # a linear density field comes out exact at every located pixel
    def prim(x):
        W = np.zeros(x.shape[:-1] + (5,))
        W[..., 0] = 1.0 + 0.05 * x[..., 0] - 0.02 * x[..., 1]
        W[..., 4] = 1.0
        return W
    r.render(solver.state_blocks_from_primitive_function(op, prim), mode=1)
    grid = r._grid.cpu().numpy().reshape(-1, 5)
    ok = r.pixel_block >= 0
    expect = 1.0 + 0.05 * r.pixel_points[:, 0] - 0.02 * r.pixel_points[:, 1]
    assert np.max(np.abs(grid[ok, 0] - expect[ok])) < 1e-6
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record()
    for _ in range(20):
        r.render(states, mode=0)
    stop.record()
    torch.cuda.synchronize()
    assert start.elapsed_time(stop) / 20 < 10.0
