"""Synthetic workloads of the benchmark configurations besides the sphere: the Taylor-Green
vortex (periodic hexahedron box) and the isentropic vortex on hybrid meshes (order of
accuracy).  Non-dimensional with rho_inf = p_inf = 1 and gas constant 1 (c_inf = sqrt(gamma)).
"""

import time

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
    out = []
    for bp, block in zip(plan.blocks, plan.mesh.element_blocks):
        geo, xyz = plan.mesh.geometry(block)
        xq = np.einsum("qi,eid->eqd", geo.basis(bp.ref.points), xyz)
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
               radius=0.1, autotune=True, tensor_cores=False):
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
        tc_blocks = op.native.set_tensor_cores(True) if tensor_cores and precision == "mixed" else 0
        states = {k: v.clone() for k, v in start.items()}
        widths = op.autotune(states) if autotune else None
        integ = HybridSSPRK3(op, cfl=cfl, graph=graph)
        first = integ.checked_step_inplace(states, dt).view(torch.int32)[0] != 0     # the graph capture
        ok, seconds = _timed(lambda: advance(integ, states, steps - 1, dt))
        err = l2_density_error(op, states, lambda x: vortex_primitive(x, t_end, radius=radius, length=length))
        err /= length ** 1.5
        out.append(dict(n=n, degree=degree, precision=precision, cfl=cfl, radius=radius,
                        elements={bp.etype: bp.E for bp in op.plan.blocks},
                        dofs=dof_count(op), steps=steps, dt=dt, admissible=ok and bool(first.item()),
                        l2_density=err, seconds=seconds, dof_updates_per_s=dof_count(op) * (steps - 1) / seconds,
                        widths=widths, tensor_core_blocks=tc_blocks))
        del states, integ
    return out


def run_tgv(n=16, degree=2, steps=10, cfl=0.3, precision="float64", graph=False):
    """The Taylor-Green configuration: ``steps`` checked steps at the stable dt of each step, timed
    with CUDA events after two untimed steps on a copy of the start."""
    import torch
    from .time_integration import HybridSSPRK3
    solver, op, states = tgv_case(n, degree, precision=precision)
    integ = HybridSSPRK3(op, cfl=cfl, graph=graph)
    spare = {k: v.clone() for k, v in states.items()}
    for _ in range(2):                       # untimed: module load and first launches
        integ.checked_step_inplace(spare, float(integ.stable_dt_device(spare).item()))
    del spare

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
    [--precision float64,mixed] | tgv [--n 16] [--degree 2] [--steps 10] | reacting [--scale full]
    [--degree 2] [--steps 10] | ensemble [--cases 64] [--elements 5000,60000] [--steps 10]: one
    JSON line per run, and for the vortex the observed orders between consecutive sizes."""
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m jax_fluid_sim_b200.workloads")
    ap.add_argument("case", choices=["vortex", "tgv", "reacting", "ensemble", "learned"])
    ap.add_argument("--limiter", default="mood", choices=["mood", "positivity"])
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--eval-steps", type=int, default=2000)
    ap.add_argument("--threshold", type=float, default=0.5)
    ap.add_argument("--tensor-cores", type=int, default=0, help="vortex: mixed runs on the tensor-core volume kernel")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--elements", default="5000,60000")
    ap.add_argument("--scale", default="full")
    ap.add_argument("--sizes", default="8,16,32")
    ap.add_argument("--degrees", default="1,2,3")
    ap.add_argument("--precision", default="float64,mixed")
    ap.add_argument("--cfl", type=float, default=0.3)
    ap.add_argument("--periods", type=float, default=1.0)
    ap.add_argument("--radius", type=float, default=0.1)
    ap.add_argument("--autotune", type=int, default=1, help="time the dense kernels' launch shapes first")
    ap.add_argument("--n", type=int, default=16)
    ap.add_argument("--degree", type=int, default=2)
    ap.add_argument("--steps", type=int, default=10)
    args = ap.parse_args(argv)
    precisions = args.precision.split(",")
    if args.case == "learned":
        print(json.dumps(run_learned(args.scale, args.train_steps, args.eval_steps, threshold=args.threshold,
                                     precision=precisions[-1])), flush=True)
        return
    if args.case == "ensemble":
        lo, hi = (float(x) for x in args.elements.split(","))
        groups, total = run_ensemble(args.cases, (lo, hi), args.steps, precision=precisions[0], cfl=args.cfl,
                                     limiter=args.limiter)
        for g in groups:
            print(json.dumps(g), flush=True)
        print(json.dumps(total), flush=True)
        return
    if args.case == "reacting":
        for r in run_reacting(args.scale, args.degree, args.steps, precisions=precisions, cfl=args.cfl):
            print(json.dumps(r), flush=True)
        return
    if args.case == "tgv":
        for prec in precisions:
            print(json.dumps(run_tgv(args.n, args.degree, args.steps, args.cfl, prec)), flush=True)
        return
    sizes = [int(s) for s in args.sizes.split(",")]
    for degree in (int(d) for d in args.degrees.split(",")):
        errors = {}
        for n in sizes:
            for r in run_vortex(n, degree, precisions, args.cfl, periods=args.periods, radius=args.radius,
                                autotune=bool(args.autotune), tensor_cores=bool(args.tensor_cores)):
                prev = errors.get(r["precision"])
                if prev is not None:
                    r["order"] = float(np.log(prev[1] / r["l2_density"]) / np.log(n / prev[0]))
                errors[r["precision"]] = (n, r["l2_density"])
                print(json.dumps(r), flush=True)



# --------------------------------------------------------------------------- Mach-3 sphere
SPHERE_GAMMA, SPHERE_MACH, SPHERE_RE, SPHERE_T_INF, SPHERE_T_WALL = 1.4, 3.0, 1.0e5, 220.0, 300.0


def sphere_mesh(scale="full"):
    """O/H sphere grids of the Mach-3 configuration: "full" 202,752 hexahedra, "medium" 39,488,
    "small" and "tiny" for tests."""
    if scale == "full":
        return meshgen.sphere_oh_grid()
    if scale == "medium":
        return meshgen.sphere_oh_grid(n=16, n_radial=10, outer=((4, 16), (6, 6), (6, 6)))
    if scale == "small":
        return meshgen.sphere_oh_grid(n=8, n_radial=6, outer=((3, 10), (4, 4), (4, 4)))
    return meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))


def sphere_shock_state(solver, op, u, gamma=SPHERE_GAMMA, mach=SPHERE_MACH, radius=0.65):
    """The Mach-3 normal-shock (Rankine-Hugoniot) state in the elements whose centroid lies inside
    r < radius, the free stream (rho = p = 1, velocity u along x) in the others; each element
    starts constant, so the jump sits on element faces."""
    g, M = gamma, mach
    rho2 = (g + 1) * M ** 2 / ((g - 1) * M ** 2 + 2)
    p2 = 1 + 2 * g / (g + 1) * (M ** 2 - 1)

    def prim(xyz):
        inside = np.broadcast_to(np.linalg.norm(xyz.mean(axis=1), axis=-1)[:, None] < radius, xyz.shape[:-1])
        W = np.zeros(xyz.shape[:-1] + (5,))
        W[..., 0] = np.where(inside, rho2, 1.0)
        W[..., 1] = np.where(inside, u / rho2, u)
        W[..., 4] = np.where(inside, p2, 1.0)
        return W

    return solver.state_blocks_from_primitive_function(op, prim)


def sphere_case(scale="full", degree=3, precision="mixed"):
    """Solver, Navier-Stokes operator, boundary descriptor and shocked start of the Mach-3 viscous
    sphere (Re_D = 1e5, isothermal wall 300 K / 220 K), non-dimensional as the reference driver
    (rho = p = 1, U = 3 sqrt(gamma), mu = U / Re)."""
    from .boundary import FarfieldWallBoundary
    from .mesh import HybridMesh
    from .operators import HybridNavierStokesOperator
    from .solver import HybridCompressibleSolver
    u = SPHERE_MACH * np.sqrt(SPHERE_GAMMA)
    solver = HybridCompressibleSolver(HybridMesh(sphere_mesh(scale)), polynomial_degree=degree,
                                      dynamic_viscosity=u / SPHERE_RE)
    op = HybridNavierStokesOperator(solver, precision=precision)
    bc = FarfieldWallBoundary(solver, np.array([1.0, u, 0.0, 0.0, 1.0]),
                              wall_temperature=SPHERE_T_WALL / SPHERE_T_INF)
    return solver, op, bc, sphere_shock_state(solver, op, u)


def run_learned(scale="full", train_steps=2000, eval_steps=2000, negative_fraction=0.01, threshold=0.5,
                epochs=4, precision="mixed", seed=0, evaluate_every=100):
    """The learned troubled-cell protocol on the Mach-3 sphere at P3 with MOOD: ``train_steps``
    plain steps from the shocked start, each labelling every element by the a-posteriori detector
    on the first SSP-RK stage (all positives and a seeded ``negative_fraction`` of the negatives
    are kept); the predictor is trained on them; then, from the state reached, ``eval_steps``
    plain steps and ``eval_steps`` learned steps (one dt for all), each run replayed as a CUDA graph
    and timed with CUDA events.  The predictor's missed-cell and false-positive rates are measured
    in evaluate mode (the plain step, every element tested, predictions only counted) on every
    ``evaluate_every``-th step of the plain run.  Returns one dict."""
    import torch
    from .limiter import HybridMOODSubcellLimiter, HybridPositivityLimiter
    from .predictor import TroubledCellPredictor
    from .time_integration import HybridSSPRK3
    solver, op, bc, U = sphere_case(scale, 3, precision)
    limiter = HybridMOODSubcellLimiter(op, positivity=HybridPositivityLimiter(op))
    integ = HybridSSPRK3(op, cfl=0.3, limiter=limiter, graph=True)
    dt = integ.stable_dt(U, bc)
    E = sum(bp.E for bp in op.plan.blocks)
    predictor = TroubledCellPredictor(op, threshold=threshold, seed=seed)
    gen = torch.Generator(device="cuda").manual_seed(seed)
    Xs, ys, flagged = [], [], []
    t0 = time.time()
    for _ in range(train_steps):
        X, y = predictor.labelled_samples(U, dt, bc, limiter)
        keep = y.bool() | (torch.rand(y.shape, generator=gen, device="cuda") < negative_fraction)
        Xs.append(X[keep])
        ys.append(y[keep])
        flagged.append(y.sum())
        integ.checked_step_inplace(U, dt, bc)
    flagged = torch.stack(flagged).double().cpu().numpy() / E
    X, y = torch.cat(Xs), torch.cat(ys)
    del Xs, ys
    history = predictor.fit(X, y, epochs=epochs, batch=8192)
    train_s = time.time() - t0
    start = {k: v.clone() for k, v in U.items()}

    def run(mode):
        predictor.attach(mode)
        predictor.counts(reset=True)
        cur = {k: v.clone() for k, v in start.items()}
        ok = torch.ones((), dtype=torch.bool, device="cuda")
        ok &= integ.checked_step_inplace(cur, dt, bc).view(torch.int32)[0] != 0     # graph capture
        t_start, t_stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_start.record()
        for k in range(1, eval_steps):
            ok &= integ.checked_step_inplace(cur, dt, bc).view(torch.int32)[0] != 0
        t_stop.record()
        torch.cuda.synchronize()
        counts = predictor.counts(reset=True)
        predictor.attach("off")
        return cur, bool(ok.item()), t_start.elapsed_time(t_stop) / 1e3, counts

    plain, plain_ok, plain_s, _ = run("off")
    learned, learned_ok, learned_s, learned_counts = run("learned")
    # predictor quality: evaluate mode on every evaluate_every-th step of a plain run
    predictor.attach("evaluate")
    predictor.counts(reset=True)
    cur = {k: v.clone() for k, v in start.items()}
    integ_eval = HybridSSPRK3(op, cfl=0.3, limiter=limiter, graph=False)
    hit = missed = fp = predicted = steps_eval = 0
    for k in range(eval_steps):
        if k % evaluate_every == 0:
            predictor.attach("evaluate")
            integ_eval.checked_step_inplace(cur, dt, bc)
            c = predictor.counts(reset=True)
            hit, missed, fp, predicted = hit + c["hit"], missed + c["missed"], fp + c["false_positive"], \
                predicted + c["predicted"]
            steps_eval += 1
            predictor.attach("off")
        else:
            integ.checked_step_inplace(cur, dt, bc)
    num = sum(float(((learned[k][..., 0] - plain[k][..., 0]) ** 2).sum()) for k in plain)
    den = sum(float((plain[k][..., 0] ** 2).sum()) for k in plain)
    dofs = dof_count(op)
    positives = hit + missed
    return dict(case="learned", scale=scale, elements=E, dofs=dofs, precision=precision, dt=dt,
                train_steps=train_steps, eval_steps=eval_steps, samples=int(X.shape[0]),
                positives_in_samples=int(y.sum().item()), negative_fraction=negative_fraction,
                threshold=threshold, epochs=epochs, loss_first_last=[history[0], history[-1]],
                train_seconds=round(train_s, 1),
                flagged_fraction_per_stage={"mean": float(flagged.mean()), "min": float(flagged.min()),
                                            "max": float(flagged.max())},
                plain={"dof_updates_per_s": dofs * (eval_steps - 1) / plain_s, "admissible": plain_ok},
                learned={"dof_updates_per_s": dofs * (eval_steps - 1) / learned_s, "admissible": learned_ok,
                         "predicted_per_stage": learned_counts["predicted"] / max(3 * (eval_steps), 1),
                         "missed_caught_by_detector_per_stage": learned_counts["missed"] / max(3 * eval_steps, 1)},
                evaluate={"steps": steps_eval, "missed_rate": missed / max(positives, 1),
                          "false_positive_rate": fp / max(3 * steps_eval * E - positives, 1),
                          "detector_flags_per_stage": positives / max(3 * steps_eval, 1),
                          "predicted_per_stage": predicted / max(3 * steps_eval, 1)},
                density_l2_rel_learned_vs_plain=(num / den) ** 0.5)


# --------------------------------------------------------------------------- reacting sphere
REACTING_MACH, REACTING_T_INF, REACTING_P_INF, REACTING_T_WALL = 8.0, 220.0, 500.0, 300.0
AIR_MASS_FRACTIONS = {"N2": 0.767, "O2": 0.233}


def reacting_farfield(mach=REACTING_MACH, gamma=1.4):
    """Free stream [rho, u, v, w, p, Y(e-, N+, O+, NO+, N2+, O2+, N, O, NO, N2, O2)] in the
    reference driver's units (rho = p = 1, gas constant 1, u = M sqrt(gamma);
    run_hybrid_sphere.py:79-91,107-108)."""
    W = np.zeros(16)
    W[0], W[1], W[4] = 1.0, mach * np.sqrt(gamma), 1.0
    W[5 + 9], W[5 + 10] = AIR_MASS_FRACTIONS["N2"], AIR_MASS_FRACTIONS["O2"]
    return W


def reacting_mesh(scale="full"):
    """O/H sphere grids of radius 0.5 (0.1 m): "full" about 150k hexahedra."""
    if scale == "full":
        return meshgen.sphere_oh_grid(n=22, n_radial=18, outer=((7, 28), (10, 10), (10, 10)))
    if scale == "small":
        return meshgen.sphere_oh_grid(n=8, n_radial=6, outer=((3, 10), (4, 4), (4, 4)))
    return meshgen.sphere_oh_grid(n=4, n_radial=2, outer=((1, 3), (1, 1), (1, 1)))


def reacting_case(scale="full", degree=2, reynolds=2.6e5, precision="float64", mach=REACTING_MACH, gamma=1.4):
    """Mach-8 viscous flow past the sphere with the 11 Air-11 species carried as conserved
    variables: solver, Navier-Stokes operator, boundary (isothermal 300 K wall), coupler and the
    shocked start (the normal-shock state in the elements whose centroid lies inside r < 0.65,
    the free stream elsewhere; species at the free-stream fractions).  Re_D = 2.6e5 is the
    Reynolds number of 500 Pa, 220 K air past a 0.2 m sphere at Mach 8; the coupler's length
    unit is 0.2 m (the grid's sphere diameter is 1)."""
    from .air11 import AIR11_SPECIES
    from .boundary import FarfieldWallBoundary
    from .chemistry import ReactingFlowCoupler
    from .mesh import HybridMesh
    from .operators import HybridNavierStokesOperator
    from .solver import HybridCompressibleSolver
    far = reacting_farfield(mach, gamma)
    mu = far[1] / reynolds
    solver = HybridCompressibleSolver(HybridMesh(reacting_mesh(scale)), species_names=tuple(s.name for s in AIR11_SPECIES),
                                      gamma=gamma, polynomial_degree=degree, dynamic_viscosity=mu)
    op = HybridNavierStokesOperator(solver, precision=precision)
    bc = FarfieldWallBoundary(solver, far, wall_temperature=REACTING_T_WALL / REACTING_T_INF)
    coupler = ReactingFlowCoupler(dimensionless=True, reference_temperature=REACTING_T_INF,
                                  reference_pressure=REACTING_P_INF, reference_length=0.2, gamma=gamma)
    return solver, op, bc, coupler, solver.state_blocks_from_primitive_function(
        op, lambda xyz: reacting_start(xyz, mach, gamma))


def reacting_start(xyz, mach=REACTING_MACH, gamma=1.4):
    """Primitive start of the reacting sphere at the solution nodes xyz (E, N, 3): the normal-shock
    state in the elements whose centroid lies inside r < 0.65, the free stream elsewhere, species
    at the free-stream fractions."""
    far = reacting_farfield(mach, gamma)
    rho2 = (gamma + 1) * mach ** 2 / ((gamma - 1) * mach ** 2 + 2)
    p2 = 1 + 2 * gamma / (gamma + 1) * (mach ** 2 - 1)
    inside = np.broadcast_to(np.linalg.norm(xyz.mean(axis=1), axis=-1)[:, None] < 0.65, xyz.shape[:-1])
    W = np.broadcast_to(far, xyz.shape[:-1] + (16,)).copy()
    W[..., 0] = np.where(inside, rho2, 1.0)
    W[..., 1] = np.where(inside, far[1] / rho2, far[1])
    W[..., 4] = np.where(inside, p2, 1.0)
    return W


def stagnation_shock_x(node_xyz, rho, radius=0.5):
    """Shock position on the stagnation line (the negative x axis upstream of a sphere of the given
    radius centred at the origin): walking downstream from the far field over the solution nodes
    that lie on the axis (nodes shared by elements averaged), the x where the density first reaches
    the midpoint between its far-field value and its largest value on the line, interpolated
    linearly between the two nodes that bracket it; NaN while the line holds no compression (its
    largest density within 1e-6 of the far-field one).  node_xyz (E, N, 3), rho (E, N) numpy."""
    on = (np.hypot(node_xyz[..., 1], node_xyz[..., 2]) < 1e-9) & (node_xyz[..., 0] <= -radius)
    x = np.round(node_xyz[..., 0][on], 12)
    xs, inv = np.unique(x, return_inverse=True)
    r = np.bincount(inv, weights=rho[on]) / np.bincount(inv)
    if r.max() <= r[0] * (1.0 + 1e-6):
        return float("nan")
    mid = 0.5 * (r[0] + r.max())
    k = int(np.argmax(r >= mid))
    return float(xs[k - 1] + (mid - r[k - 1]) / (r[k] - r[k - 1]) * (xs[k] - xs[k - 1]))


def species_closure(states):
    """max over nodes of |sum_s rho_s - rho| / rho: the species densities' sum against the mixture
    density (both conserved; the flux and the coupler keep them equal to round-off)."""
    worst = 0.0
    for U in states.values():
        rho = U[..., 0]
        worst = max(worst, float(((U[..., 5:].sum(-1) - rho).abs() / rho).max()))
    return worst


def run_reacting(scale="full", degree=2, steps=10, warmup=3, precisions=("float64", "mixed"), cfl=0.3):
    """The reacting-sphere configuration: each step is one checked SSP-RK3 step with the MOOD
    limiter (replayed as a CUDA graph) followed by the operator-split Air-11 source on every
    block (run_hybrid_sphere.py:292-312).  From the shocked start, ``warmup`` steps, then
    ``steps`` timed steps per precision from the same state and dt; returns DOF-updates/s,
    the flow and chemistry shares, the species closure and the density L2 difference of each
    run to the float64 run."""
    import torch
    from .limiter import HybridMOODSubcellLimiter, HybridPositivityLimiter
    from .time_integration import HybridSSPRK3
    solver, op64, bc, coupler, start = reacting_case(scale, degree)

    def integrator(op):
        lim = HybridMOODSubcellLimiter(op, positivity=HybridPositivityLimiter(op))
        return HybridSSPRK3(op, cfl=cfl, limiter=lim, graph=True)

    integ = integrator(op64)
    dt = integ.stable_dt(start, bc)
    for _ in range(warmup):
        integ.checked_step_inplace(start, dt, bc)
        for k in start:
            coupler.react_block(start[k], dt, out=start[k])
    torch.cuda.synchronize()
    out, plain = [], None
    for precision in precisions:
        op = op64 if precision == "float64" else op64.with_precision(precision)
        it = integ if precision == "float64" else integrator(op)
        U = {k: v.clone() for k, v in start.items()}
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * steps + 1)]
        ok = torch.ones((), dtype=torch.bool, device="cuda")
        torch.cuda.synchronize()
        ev[0].record()
        for s in range(steps):
            ok &= it.checked_step_inplace(U, dt, bc).view(torch.int32)[0] != 0
            ev[2 * s + 1].record()
            for k in U:
                coupler.react_block(U[k], dt, out=U[k])
            ev[2 * s + 2].record()
        torch.cuda.synchronize()
        total = ev[0].elapsed_time(ev[-1]) * 1e-3
        chem = sum(ev[2 * s + 1].elapsed_time(ev[2 * s + 2]) for s in range(steps)) * 1e-3
        r = dict(precision=precision, elements=sum(bp.E for bp in op.plan.blocks), dofs=dof_count(op), steps=steps,
                 dt=dt, admissible=bool(ok.item()), seconds=total, chemistry_seconds=chem,
                 dof_updates_per_s=dof_count(op) * steps / total, species_closure=species_closure(U))
        if plain is None:
            plain = U
        else:
            num = sum(float(((U[k][..., 0] - plain[k][..., 0]) ** 2).sum()) for k in U)
            den = sum(float((plain[k][..., 0] ** 2).sum()) for k in U)
            r["density_l2_vs_float64"] = (num / den) ** 0.5
        out.append(r)
    return out


# --------------------------------------------------------------------------- cylinder ensembles
def ensemble_cases(num_cases=64, elements=(5000, 60000), seed=0, degrees=(2, 3)):
    """Seeded cases of extruded cylinder O-grids: element count uniform in ``elements``
    (n_theta ~ 3 n_radial), free-stream Mach uniform in [0.3, 4], Re_D log-uniform in
    [1e2, 1e5], degree drawn from ``degrees``."""
    rng = np.random.default_rng(seed)
    E = rng.uniform(*elements, size=num_cases)
    mach = rng.uniform(0.3, 4.0, num_cases)
    re = 10.0 ** rng.uniform(2.0, 5.0, num_cases)
    deg = rng.choice(np.asarray(degrees), num_cases)
    out = []
    for c in range(num_cases):
        n_radial = max(4, int(round(np.sqrt(E[c] / 3.0))))
        n_theta = max(8, int(round(E[c] / n_radial / 4.0)) * 4)
        out.append(dict(n_theta=n_theta, n_radial=n_radial, mach=float(mach[c]), reynolds=float(re[c]),
                        degree=int(deg[c])))
    return out


def _cylinder_case(case, gamma=1.4):
    far = np.array([1.0, case["mach"] * np.sqrt(gamma), 0.0, 0.0, 1.0])
    return meshgen.cylinder_o_grid(case["n_theta"], case["n_radial"]), far, far[1] / case["reynolds"]


# device bytes per element of a viscous hexahedron ensemble plan and its step buffers (measured
# about 52 KB at P2 in float64 and 63 KB in mixed precision; P3 scales with the node count), with
# room for the step's buffers
ENSEMBLE_BYTES_PER_ELEMENT = {1: 40e3, 2: 80e3, 3: 170e3}


def run_ensemble(num_cases=64, elements=(5000, 60000), steps=10, warmup=2, seed=0, precision="float64", cfl=0.3,
                 limiter="mood"):
    """The ensemble configuration: the cases of ``ensemble_cases`` grouped by degree, each group
    one HybridEnsemble (one launch per kernel per RK stage for all its cases, the step replayed
    as a CUDA graph), against the same cases solved one after another on their own plans, at the
    same dt and step count (checked SSP-RK3 with the MOOD limiter, or with ``limiter="positivity"``
    the positivity limiter alone, which needs no subcell tables).  Returns per group and in total
    the DOF-updates/s of both, timed with CUDA events after ``warmup`` untimed steps."""
    import gc
    import torch
    from .ensemble import HybridEnsemble
    from .limiter import HybridMOODSubcellLimiter, HybridPositivityLimiter
    from .time_integration import HybridSSPRK3
    from .boundary import FarfieldWallBoundary
    from .mesh import HybridMesh
    from .operators import HybridNavierStokesOperator
    from .solver import HybridCompressibleSolver

    def integrator(op):
        pos = HybridPositivityLimiter(op)
        lim = HybridMOODSubcellLimiter(op, positivity=pos) if limiter == "mood" else pos
        return HybridSSPRK3(op, cfl=cfl, limiter=lim, graph=True)

    def timed_steps(it, U, dt, bc):
        for _ in range(warmup):
            it.checked_step_inplace(U, dt, bc)
        return _timed(lambda: [it.checked_step_inplace(U, dt, bc) for _ in range(steps)])[1]

    cases = ensemble_cases(num_cases, elements, seed)
    groups, total = [], dict(dofs=0, ensemble_seconds=0.0, sequential_seconds=0.0)
    for degree in sorted({c["degree"] for c in cases}):
        members = [c for c in cases if c["degree"] == degree]
        built = [_cylinder_case(c) for c in members]
        # one ensemble per group when its plan fits the device, else consecutive sub-ensembles that
        # do (device bytes per element of a viscous hexahedron plan at this degree, with margin)
        budget = 0.7 * torch.cuda.mem_get_info()[0] / ENSEMBLE_BYTES_PER_ELEMENT[degree]
        chunks, cur, size = [], [], 0
        for b, c in zip(built, members):
            n = c["n_theta"] * c["n_radial"]
            if cur and size + n > budget:
                chunks.append(cur)
                cur, size = [], 0
            cur.append(b)
            size += n
        chunks.append(cur)
        # one dt for the whole group: the smallest stable dt of its sub-ensembles
        ens_list, plan_gb = [], 0.0
        dt = float("inf")
        for part in chunks:
            free0 = torch.cuda.mem_get_info()[0]
            ens = HybridEnsemble([b[0] for b in part], [b[1] for b in part], [b[2] for b in part],
                                 polynomial_degree=degree, precision=precision)
            U = ens.freestream_states()
            plan_gb = max(plan_gb, (free0 - torch.cuda.mem_get_info()[0]) / 1e9)
            it = integrator(ens.operator)
            dt = min(dt, it.stable_dt(U, ens.boundary))
            if len(chunks) == 1:
                ens_list.append((ens, U, it))
            del ens, U, it
            gc.collect()
        t_ens, dofs = 0.0, 0
        for part in chunks:
            if len(chunks) == 1:
                ens, U, it = ens_list.pop()
            else:
                ens = HybridEnsemble([b[0] for b in part], [b[1] for b in part], [b[2] for b in part],
                                     polynomial_degree=degree, precision=precision)
                U = ens.freestream_states()
                it = integrator(ens.operator)
            t_ens += timed_steps(it, U, dt, ens.boundary)
            dofs += ens.dofs
            del ens, U, it
            gc.collect()
            torch.cuda.empty_cache()
        t_seq, ok = 0.0, True
        for src, far, mu in built:
            solver = HybridCompressibleSolver(HybridMesh(src), polynomial_degree=degree, dynamic_viscosity=mu)
            op = HybridNavierStokesOperator(solver, precision=precision)
            bc = FarfieldWallBoundary(solver, far)
            Uc = solver.uniform_state_blocks(far[0], far[1:4], far[4])
            t_seq += timed_steps(integrator(op), Uc, dt, bc)
            del solver, op, Uc
            gc.collect()                  # free the case's device plan before the next one
        groups.append(dict(degree=degree, cases=len(members), limiter=limiter, precision=precision,
                           elements=int(sum(c["n_theta"] * c["n_radial"] for c in members)), ensembles=len(chunks),
                           dofs=dofs, dt=dt, device_gb=round(plan_gb, 2), ensemble_dof_updates_per_s=dofs * steps / t_ens,
                           sequential_dof_updates_per_s=dofs * steps / t_seq, speedup=t_seq / t_ens))
        total["dofs"] += dofs
        total["ensemble_seconds"] += t_ens
        total["sequential_seconds"] += t_seq
        gc.collect()
        torch.cuda.empty_cache()
    total.update(steps=steps, ensemble_dof_updates_per_s=total["dofs"] * steps / total["ensemble_seconds"],
                 sequential_dof_updates_per_s=total["dofs"] * steps / total["sequential_seconds"],
                 speedup=total["sequential_seconds"] / total["ensemble_seconds"])
    return groups, total


if __name__ == "__main__":
    main()
