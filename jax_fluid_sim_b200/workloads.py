"""Synthetic workloads of the benchmark configurations besides the sphere: the Taylor-Green
vortex (periodic hexahedron box) and the isentropic vortex on hybrid meshes (order of
accuracy).  Non-dimensional with rho_inf = p_inf = 1 and gas constant 1 (c_inf = sqrt(gamma)).
"""

import numpy as np

from . import meshgen


def tgv_mesh(n=16, jitter=0.0, seed=0):
    """[0, 2 pi]^3, n^3 hexahedra, periodic in all three directions."""
    return meshgen.box_hex((n, n, n), lo=(0.0, 0.0, 0.0), hi=(2 * np.pi,) * 3, jitter=jitter, seed=seed,
                           periodic=(True, True, True))


def tgv_primitive(xyz, mach=0.1, gamma=1.4):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0, rho = 1,
    p = p0 + (rho / 16)(cos 2x + cos 2y)(cos 2z + 2), p0 = 1 / (gamma M^2)."""
    x, y, z = xyz[..., 0], xyz[..., 1], xyz[..., 2]
    W = np.zeros(xyz.shape[:-1] + (5,))
    W[..., 0] = 1.0
    W[..., 1] = np.sin(x) * np.cos(y) * np.cos(z)
    W[..., 2] = -np.cos(x) * np.sin(y) * np.cos(z)
    W[..., 4] = 1.0 / (gamma * mach ** 2) + (np.cos(2 * x) + np.cos(2 * y)) * (np.cos(2 * z) + 2.0) / 16.0
    return W


def vortex_velocity(mach=0.5, gamma=1.4):
    """Free stream along (1, 1, 1) at the given Mach number."""
    return mach * np.sqrt(gamma) * np.ones(3) / np.sqrt(3.0)


def vortex_period(mach=0.5, gamma=1.4, length=1.0):
    """Time for the vortex to come back to its start in the periodic box of side ``length``."""
    return length / vortex_velocity(mach, gamma)[0]


def vortex_primitive(xyz, t=0.0, beta=5.0, radius=0.1, mach=0.5, gamma=1.4, center=(0.5, 0.5), length=1.0):
    """Isentropic vortex of strength beta (axis along z), advected by the free stream of
    ``vortex_velocity`` through the periodic box [0, length]^3; ``radius`` and ``center`` are in
    units of the box side.  u = U - beta/(2 pi) f y', v = V + beta/(2 pi) f x',
    T = 1 - (gamma-1) beta^2 / (8 gamma pi^2) f^2, rho = T^(1/(gamma-1)), p = rho T, with
    f = exp((1 - r^2)/2), (x', y') the nearest-image offsets from the moved centre in units of
    the radius and r^2 = x'^2 + y'^2.  Radius 0.1 is Shu's vortex (radius 1 in a box of side 10);
    f r is 3e-5 at the half-box distance, the size of the nearest-image field's kink across the
    periodic seams."""
    U = vortex_velocity(mach, gamma)
    cx = (center[0] + U[0] * t / length) % 1.0
    cy = (center[1] + U[1] * t / length) % 1.0
    dx = (xyz[..., 0] / length - cx + 0.5) % 1.0 - 0.5
    dy = (xyz[..., 1] / length - cy + 0.5) % 1.0 - 0.5
    xb, yb = dx / radius, dy / radius
    r2 = xb ** 2 + yb ** 2
    f = np.exp(0.5 * (1.0 - r2))
    T = 1.0 - (gamma - 1.0) * beta ** 2 / (8.0 * gamma * np.pi ** 2) * f ** 2
    W = np.zeros(xyz.shape[:-1] + (5,))
    W[..., 0] = T ** (1.0 / (gamma - 1.0))
    W[..., 1] = U[0] - beta / (2 * np.pi) * f * yb
    W[..., 2] = U[1] + beta / (2 * np.pi) * f * xb
    W[..., 3] = U[2]
    W[..., 4] = W[..., 0] * T
    return W


def quadrature_points(plan):
    """Physical quadrature points (E, Nq, 3) and weights w_q |J| (E, Nq) of every element block."""
    from .reference import RefElement
    out = []
    for bp, block in zip(plan.blocks, plan.mesh.element_blocks):
        xyz = plan.mesh.points[block.connectivity]
        xq = np.einsum("qi,eid->eqd", RefElement(bp.etype, 1).basis(bp.ref.points), xyz)
        out.append((xq, bp.wdet))
    return out


def l2_density_error(operator, states, primitive):
    """sqrt(sum over elements and quadrature points of w_q |J| (rho_h - rho)^2), rho from
    ``primitive(xyz)[..., 0]``; the discrete density is the nodal state through the basis."""
    total = 0.0
    for (xq, wdet), name, bp in zip(quadrature_points(operator.plan), operator.names, operator.plan.blocks):
        U = states[name]
        rho = U[..., 0].detach().cpu().numpy() if hasattr(U, "detach") else np.asarray(U)[..., 0]
        diff = np.einsum("qn,en->eq", bp.ref.B, rho) - primitive(xq)[..., 0]
        total += float(np.sum(wdet * diff * diff))
    return np.sqrt(total)


def tgv_case(n=16, degree=2, mach=0.1, reynolds=1600.0, prandtl=0.71, gamma=1.4, precision="float64",
             jitter=0.0, seed=0):
    """Solver, Navier-Stokes operator and device state of the Taylor-Green vortex (rho0 = U0 = L = 1,
    mu = 1/Re, gas constant 1)."""
    from .mesh import HybridMesh
    from .operators import HybridNavierStokesOperator
    from .solver import HybridCompressibleSolver
    solver = HybridCompressibleSolver(HybridMesh(tgv_mesh(n, jitter, seed)), gamma=gamma, polynomial_degree=degree,
                                      dynamic_viscosity=1.0 / reynolds, prandtl=prandtl)
    op = HybridNavierStokesOperator(solver, precision=precision)
    states = solver.state_blocks_from_primitive_function(op, lambda x: tgv_primitive(x, mach, gamma))
    return solver, op, states


def vortex_case(n=8, degree=2, jitter=0.1, seed=0, precision="float64", length=1.0, **vortex):
    """Solver, Euler operator and device state of the isentropic vortex on ``meshgen.hybrid_box``
    of n^3 cubes with side ``length``.

    The reference scales the inverse mass matrix of every element below an absolute volume of
    1e-4 by V / 1e-4 (hybrid/geometry.py:189-192).  In the unit cube the tetrahedra of 16^3 and
    32^3 cubes fall below it and the scheme loses consistency there, so order studies use a box
    of side 10 (every element above the floor): the unit cube in units of a tenth of its side."""
    from .mesh import HybridMesh
    from .operators import HybridEulerOperator
    from .solver import HybridCompressibleSolver
    solver = HybridCompressibleSolver(HybridMesh(meshgen.hybrid_box((n, n, n), hi=(length,) * 3, jitter=jitter,
                                                                    seed=seed)),
                                      gamma=vortex.get("gamma", 1.4), polynomial_degree=degree)
    op = HybridEulerOperator(solver, precision=precision)
    states = solver.state_blocks_from_primitive_function(
        op, lambda x: vortex_primitive(x, 0.0, length=length, **vortex))
    return solver, op, states


def dof_count(operator):
    return sum(bp.E * bp.Np for bp in operator.plan.blocks)


def convective_dt(operator, states, cfl):
    """cfl / max over elements of (2P + 1) max(|u| + c) / h, h the reference's characteristic
    length (time_integration.py:49-91) -- the convective limit of the reference's stable dt
    without its clamp to [1e-7, 1e-3], which would set the step of every resolution alike."""
    P, gamma = operator.plan.degree, operator.solver.gamma
    rate = 0.0
    for name, bp in zip(operator.names, operator.plan.blocks):
        U = states[name].detach().cpu().numpy() if hasattr(states[name], "detach") else np.asarray(states[name])
        rho = U[..., 0]
        vel = U[..., 1:4] / rho[..., None]
        p = (gamma - 1.0) * (U[..., 4] - 0.5 * rho * np.sum(vel * vel, axis=-1))
        speed = np.linalg.norm(vel, axis=-1) + np.sqrt(gamma * p / rho)
        rate = max(rate, float(np.max((2 * P + 1) * speed.max(axis=1) / bp.length)))
    return cfl / rate


def advance(integrator, states, steps, dt):
    """``steps`` checked SSP-RK3 steps of size dt in place; True when every step was admissible."""
    import torch
    ok = torch.ones((), dtype=torch.bool, device="cuda")
    for _ in range(steps):
        status = integrator.checked_step_inplace(states, dt)
        ok &= status.view(torch.int32)[0] != 0
    return bool(ok.item())


def equal_steps(t_end, dt_max):
    """(steps, dt): the fewest equal steps of at most dt_max that reach t_end."""
    steps = int(np.ceil(t_end / dt_max - 1e-12))
    return steps, t_end / steps


def _timed(fn):
    import torch
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    start.record()
    out = fn()
    stop.record()
    torch.cuda.synchronize()
    return out, start.elapsed_time(stop) * 1e-3


def run_vortex(n, degree, precisions=("float64",), cfl=0.3, length=10.0, periods=1.0, graph=True, seed=0,
               radius=0.1):
    """One size of the order study: the vortex through ``periods`` periods on the n^3 hybrid box
    of side ``length``, once per precision from the same start (one host plan).  Each result
    holds the density L2 error (divided by sqrt(box volume)), the step count and the
    DOF-updates/s of the timed steps (CUDA events around all steps after the first, which
    captures the step graph)."""
    import torch
    from .time_integration import HybridSSPRK3
    solver, op64, start = vortex_case(n, degree, seed=seed, length=length, radius=radius)
    t_end = periods * vortex_period(length=length)
    steps, dt = equal_steps(t_end, convective_dt(op64, start, cfl))
    out = []
    for precision in precisions:
        op = op64 if precision == "float64" else op64.with_precision(precision)
        states = {k: v.clone() for k, v in start.items()}
        integ = HybridSSPRK3(op, cfl=cfl, graph=graph)
        first = integ.checked_step_inplace(states, dt).view(torch.int32)[0] != 0     # the graph capture
        ok, seconds = _timed(lambda: advance(integ, states, steps - 1, dt))
        err = l2_density_error(op, states, lambda x: vortex_primitive(x, t_end, radius=radius, length=length))
        err /= length ** 1.5
        out.append(dict(n=n, degree=degree, precision=precision, cfl=cfl, radius=radius,
                        elements={bp.etype: bp.E for bp in op.plan.blocks},
                        dofs=dof_count(op), steps=steps, dt=dt, admissible=ok and bool(first.item()),
                        l2_density=err, seconds=seconds, dof_updates_per_s=dof_count(op) * (steps - 1) / seconds))
        del states, integ
    return out


def run_tgv(n=16, degree=2, steps=10, cfl=0.3, precision="float64", graph=False):
    """The Taylor-Green configuration: ``steps`` checked steps at the stable dt of each step."""
    import torch
    from .time_integration import HybridSSPRK3
    solver, op, states = tgv_case(n, degree, precision=precision)
    integ = HybridSSPRK3(op, cfl=cfl, graph=graph)

    def run():
        ok = torch.ones((), dtype=torch.bool, device="cuda")
        for _ in range(steps):
            dt = integ.stable_dt_device(states)
            ok &= integ.checked_step_inplace(states, float(dt.item())).view(torch.int32)[0] != 0
        return bool(ok.item())

    ok, seconds = _timed(run)
    ke = 0.0
    for (xq, wdet), name, bp in zip(quadrature_points(op.plan), op.names, op.plan.blocks):
        Uq = np.einsum("qn,env->eqv", bp.ref.B, states[name].cpu().numpy())
        ke += float(np.sum(wdet * 0.5 * np.sum(Uq[..., 1:4] ** 2, axis=-1) / Uq[..., 0]))
    return dict(n=n, degree=degree, precision=precision, dofs=dof_count(op), steps=steps, admissible=ok,
                kinetic_energy=ke / (2 * np.pi) ** 3, seconds=seconds,
                dof_updates_per_s=dof_count(op) * steps / seconds)


def main(argv=None):
    """python -m jax_fluid_sim_b200.workloads vortex [--sizes 8,16,32] [--degrees 1,2,3]
    [--precision float64,mixed] | tgv [--n 16] [--degree 2] [--steps 10]: one JSON line per run,
    and for the vortex the observed orders between consecutive sizes."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m jax_fluid_sim_b200.workloads")
    ap.add_argument("case", choices=["vortex", "tgv"])
    ap.add_argument("--sizes", default="8,16,32")
    ap.add_argument("--degrees", default="1,2,3")
    ap.add_argument("--precision", default="float64,mixed")
    ap.add_argument("--cfl", type=float, default=0.3)
    ap.add_argument("--periods", type=float, default=1.0)
    ap.add_argument("--radius", type=float, default=0.1)
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--degree", type=int, default=2)
    ap.add_argument("--steps", type=int, default=10)
    args = ap.parse_args(argv)
    precisions = args.precision.split(",")
    if args.case == "tgv":
        for prec in precisions:
            print(json.dumps(run_tgv(args.n, args.degree, args.steps, args.cfl, prec)), flush=True)
        return
    sizes = [int(s) for s in args.sizes.split(",")]
    for degree in (int(d) for d in args.degrees.split(",")):
        errors = {}
        for n in sizes:
            for r in run_vortex(n, degree, precisions, args.cfl, periods=args.periods, radius=args.radius):
                prev = errors.get(r["precision"])
                if prev is not None:
                    r["order"] = float(np.log(prev[1] / r["l2_density"]) / np.log(n / prev[0]))
                errors[r["precision"]] = (n, r["l2_density"])
                print(json.dumps(r), flush=True)


if __name__ == "__main__":
    main()
