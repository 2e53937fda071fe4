"""Throughput benchmark of the hybrid DG residual-and-update path on B200.

Workload (the headline configuration): Mach-3 viscous flow past a sphere of radius
0.5 in the box [-4,12]x[-6,6]^2, body-fitted O/H hex grid of ~200k elements, P3
(64 nodes per element), perfect gas gamma=1.4, Re_D=1e5, T_inf=220 K, no-slip
isothermal wall T_w=300 K (non-dimensional as the reference driver does:
rho=p=1, U=3*sqrt(1.4), mu=U/Re, T_w=300/220).  One step = one checked SSP-RK3
step (three stages of inviscid HLLC + BR2 viscous residual, then per stage the MOOD
troubled-cell check, subcell finite-volume recompute of troubled elements, Zhang-Shu
positivity limiter, blend and admissibility check).  Synthetic seeded mesh (numpy
generator); the start is described below (--start uniform gives the uniform free stream).

Default flow (one state, one dt for every run):
  1. start: the Mach-3 normal-shock state in the elements inside r < 0.65 around the sphere,
     free stream in the others (the jump sharpens inside elements, so MOOD has work);
  2. 20 plain steps, labelling every element by the a-posteriori detector on the first
     SSP-RK stage; the troubled-cell predictor is trained on those samples;
  3. from the state reached, three timed runs of K steps: plain float64, mixed precision
     (float32 arithmetic in the traces, BR2-lift, volume and finalize kernels; state, face
     fluxes, limiters and reductions float64), and learned + mixed (predicted elements go
     straight to the subcell scheme; the detector still tests every other element);
  4. the headline value is the fastest run whose density L2 difference to the plain run
     stays within 1e-6 ("at fixed L2 error"); every run, its L2 difference and the
     predictor's missed / false-positive rates (one step in evaluate mode) ride along.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--precision both|mixed|float64] [--limiter mood|positivity]
                    [--start shock|uniform] [--learned 0|1] [--train-steps S]

Metric: DOF-updates/s = sum_b E_b*Np_b * steps / seconds (Np = element nodes).
--impl reference times the CPU oracle (a float64 numpy restatement of the
reference's JAX code, which cannot be installed here) on a bounded sample mesh
with all host threads.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "P3 DOF-updates/s at fixed L2 error, learned+mixed vs plain; % HBM roofline"
UNIT = "DOF-updates/s"
GAMMA, MACH, RE, T_INF, T_WALL = 1.4, 3.0, 1.0e5, 220.0, 300.0


def peaks():
    try:
        return json.loads((ROOT / "MEASURED_PEAKS.json").read_text()), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    def __init__(self, index=0):
        self.index, self.samples, self.proc = index, [], None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": float(self.samples[0][1]) if self.samples[0][1].replace(".", "").isdigit() else None,
                "reasons": reasons, "samples": len(self.samples)}


def max_over_ranks(value, world, device="cuda"):
    """The largest of every rank's value: a time measured on several GPUs is the slowest rank's.
    Every rank takes part and gets the result."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(scale="full"):
    from jax_fluid_sim_b200 import workloads
    return workloads.sphere_mesh(scale)


def freestream(degree):
    u = MACH * np.sqrt(GAMMA)
    return u, u * 1.0 / RE, np.array([1.0, u, 0.0, 0.0, 1.0])


def rhs_bytes(op, nv, sizeof=8):
    """Algorithmic HBM bytes of one RHS evaluation (each input read once, outputs written once):
    the whole-RHS formula with J^-1, w|J| and the inverse mass counted for the non-affine
    elements only (affine hexahedra need 11 values)."""
    total = 0
    for b, bp in enumerate(op.plan.blocks):
        Ea = getattr(op.native, "affine_count", 0) if b == 0 else 0
        total += 2 * sizeof * nv * bp.E * bp.Np             # U in, R out
        total += sizeof * 10 * (bp.E - Ea) * bp.Nq          # J^-1 (9) + w|J| (1) per volume point
        total += sizeof * (bp.E - Ea) * bp.Np * bp.Np       # dense inverse mass
        total += sizeof * 11 * Ea
    for fp in op.plan.faces.values():
        total += fp.F * (sizeof * fp.nq * (2 * nv + 4 + nv) + 8)
    return total


STAGES = ["traces", "face_flux", "lift", "volume", "face_visc", "finalize"]


def stage_bytes(op, nv, split, sizeof=8):
    """Algorithmic HBM bytes per launch of each RHS stage of the sum-factorised hex path
    (every input read once, every output written once; the device buffers are float64 in both
    precision modes)."""
    out = dict.fromkeys(STAGES, 0)
    visc = op.viscous
    for b, bp in enumerate(op.plan.blocks):
        E, Np, Nq, nlf = bp.E, bp.Np, bp.Nq, bp.nlf
        # affine hexahedra read 11 values (constant J^-1, det J, M^-1 factor) instead of the dense
        # M^-1 and the per-point metrics
        Ea = getattr(op.native, "affine_count", 0) if b == 0 else 0
        Ed = E - Ea
        nqf = max(fp.nq for fp in op.plan.faces.values())
        # U in; per face point: anchor-form U (+ v, gradients and the face inverse Jacobian) out / in
        out["traces"] += sizeof * E * (nv * Np + nlf * nqf * (nv + (16 + 9 if visc else 0)))
        if visc:
            out["lift"] += sizeof * (Ed * Np * Np + Ea * 11 + E * (2 * nlf * nqf * 12 + 12 * Np))
        out["volume"] += sizeof * (Ed * 10 * Nq + Ea * 11 + E * (nv * Np + (12 * Np if visc else 0)
                                                                  + (2 if split else 1) * nv * Np))
        out["finalize"] += sizeof * (Ed * Np * Np + Ea * 11 + E * ((2 if split else 1) * nv * Np + nlf * nqf * 2 * nv
                                                                    + 3 * nv * Np))
    for fp in op.plan.faces.values():
        # traces of both sides, n and w in; both sides' fluxes out (+ v of both sides in, BR2 jumps out)
        out["face_flux"] += fp.F * (sizeof * fp.nq * (2 * nv + 4 + 2 * nv + (8 + 12 if visc else 0)) + 8)
        if visc:
            out["face_visc"] += fp.F * sizeof * fp.nq * (2 * 4 + 2 * 12 + 2 * 12 + 4 + nv)
    return out


def stage_bytes_fused(op, nv, split, sizeof=8):
    """Algorithmic HBM bytes per launch of the fused sum-factorised hex right-hand side (traces,
    face kernel, element kernel; every input read once, every output written once).  The face
    kernel is reported as the "face_flux" stage and the element kernel (nodal lift, volume terms,
    face terms, M^-1 and the outputs) as the "volume" stage.  Mixed-precision plans read float32
    copies of M^-1 and of the per-point inverse Jacobians."""
    out = dict.fromkeys(STAGES, 0)
    visc = op.viscous
    msz = 4 if op.precision == "mixed" else sizeof
    bp = op.plan.blocks[0]
    E, Np, Nq, nlf = bp.E, bp.Np, bp.Nq, bp.nlf
    Ea = getattr(op.native, "affine_count", 0)
    Ed = E - Ea
    fp = op.plan.faces["quad"]
    nqf = fp.nq
    out["traces"] = sizeof * E * (nv * Np + nlf * nqf * (nv + (16 if visc else 0))) + (msz * E * nlf * nqf * 9 if visc else 0)
    per_point = 2 * nv + 4 + 2 * nv + ((2 * 4 + 2 * 12 + 12 + nv) if visc else 0)
    out["face_flux"] = fp.F * (sizeof * nqf * per_point + 8) + (sizeof * Ed * nlf * nqf * nqf if visc else 0)
    outputs = (2 if split else 1) * nv * Np
    out["volume"] = (sizeof * E * (nv * Np + outputs + nlf * nqf * ((12 + 2 * nv) if visc else nv))
                     + msz * Ed * (10 * Nq + Np * Np) + sizeof * 11 * Ea)
    return out


def build_integrator(jfs, op, args, wall_T):
    pos = jfs.HybridPositivityLimiter(op)
    limiter = jfs.HybridMOODSubcellLimiter(op, positivity=pos) if args.limiter == "mood" else pos
    return limiter, jfs.HybridSSPRK3(op, cfl=0.3, limiter=limiter, graph=bool(getattr(args, "graph", 0)))


def shock_layer(xyz):
    """Per element (xyz: (E, Np, 3) node positions): True where the element's centroid lies
    inside r < 0.65, the layer that starts in the post-shock state."""
    return np.broadcast_to(np.linalg.norm(xyz.mean(axis=1), axis=-1)[:, None] < 0.65, xyz.shape[:-1])


def bow_shock_state(solver, op, u):
    """Synthetic start with a shock in it: the Mach-3 normal-shock (Rankine-Hugoniot) state in the
    elements whose centroid lies inside r < 0.65 around the sphere of radius 0.5, the free stream
    in the others (workloads.sphere_shock_state).  Each element starts constant, so the jump sits
    on element faces (a jump inside a P3 element would leave negative densities at its quadrature
    points); the first steps sharpen it inside the elements next to it, which gives the MOOD
    detector work."""
    from jax_fluid_sim_b200 import workloads
    return workloads.sphere_shock_state(solver, op, u, GAMMA, MACH)


def run_ours(args):
    import ctypes

    import torch
    import torch.distributed as dist

    import jax_fluid_sim_b200 as jfs
    from jax_fluid_sim_b200 import _native as N
    from jax_fluid_sim_b200.operators import _stream_ptr
    from jax_fluid_sim_b200.predictor import TroubledCellPredictor

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    t_setup = time.time()
    src = workload(args.scale)
    u, mu, farfield = freestream(3)
    solver = jfs.HybridCompressibleSolver(jfs.HybridMesh(src), polynomial_degree=args.degree, dynamic_viscosity=mu)
    precisions = {"both": ["float64", "mixed"], "float64": ["float64"], "mixed": ["mixed"]}[args.precision]
    base = jfs.HybridNavierStokesOperator(solver, precision=precisions[0])
    ops = {precisions[0]: base}
    for m in precisions[1:]:
        ops[m] = base.with_precision(m)
    bc = jfs.FarfieldWallBoundary(solver, farfield, wall_temperature=T_WALL / T_INF)
    integs = {m: build_integrator(jfs, ops[m], args, T_WALL / T_INF) for m in precisions}
    learned = args.limiter == "mood" and bool(args.learned)
    head_prec = precisions[-1]
    U0 = (bow_shock_state(solver, base, u) if args.start == "shock"
          else solver.uniform_state_blocks(1.0, [u, 0.0, 0.0], 1.0))
    dofs = sum(bp.E * bp.Np for bp in base.plan.blocks)
    E = int(sum(bp.E for bp in base.plan.blocks))
    nv = solver.layout.number_of_variables
    setup_s = time.time() - t_setup
    lim0, integ0 = integs[precisions[0]]
    dt = integ0.stable_dt(U0, bc)                   # one fixed dt for every run (same trajectory)
    # execution form of the hexahedron right-hand side per precision (fused three-launch or
    # six-launch), the faster on the start state
    forms = {m: ops[m].autotune_form(U0, bc, mood=args.limiter == "mood") for m in precisions}

    # training data: plain steps from the start, labelled by the a-posteriori detector
    predictor, train = None, None
    U_start = {k: v.clone() for k, v in U0.items()}
    if learned:
        t0 = time.time()
        predictor = TroubledCellPredictor(ops[head_prec], threshold=args.threshold)
        Xs, ys = [], []
        for _ in range(args.train_steps):
            X, y = predictor.labelled_samples(U_start, dt, bc, lim0)
            Xs.append(X)
            ys.append(y)
            integ0.checked_step_inplace(U_start, dt, bc)
        X, y = torch.cat(Xs), torch.cat(ys)
        hist = predictor.fit(X, y, epochs=args.train_epochs, batch=8192)
        torch.cuda.synchronize()
        train = {"steps": args.train_steps, "samples": int(X.shape[0]), "positives": int(y.sum().item()),
                 "epochs": args.train_epochs, "loss_first_last": [hist[0], hist[-1]],
                 "seconds": round(time.time() - t0, 1)}
        del Xs, ys, X, y

    def timed(integ, pre=None):
        Uw = {k: v.clone() for k, v in U_start.items()}
        for _ in range(args.warmup):
            integ.checked_step_inplace(Uw, dt, bc)
        del Uw
        U = {k: v.clone() for k, v in U_start.items()}
        torch.cuda.synchronize()
        if pre:
            pre()
        if world > 1:
            dist.barrier()
        start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local) as clocks:
            torch.cuda.synchronize()
            start.record()
            for _ in range(args.steps):
                integ.checked_step_inplace(U, dt, bc)
            stop.record()
            torch.cuda.synchronize()
        ms = max_over_ranks(start.elapsed_time(stop), world)
        valid, rmin, pmin = integ._status_tuple()
        return dict(ms=ms, U=U, clocks=clocks.summary(), valid=valid, rho_min=rmin, p_min=pmin,
                    value=dofs * args.steps * world / (ms / 1e3))

    runs = {}
    for m in precisions:
        runs[m] = timed(integs[m][1])
    head = head_prec
    if learned:
        predictor.attach("learned")
        runs["learned+" + head_prec] = timed(integs[head_prec][1], pre=lambda: predictor.counts(reset=True))
        in_run = predictor.counts(reset=True)
        # predictor quality on the same start: one step in evaluate mode (the plain step, every
        # element tested, the prediction only counted)
        predictor.attach("evaluate")
        Ue = {k: v.clone() for k, v in U_start.items()}
        integs[head_prec][1].checked_step_inplace(Ue, dt, bc)
        ev = predictor.counts(reset=True)
        predictor.attach("off")
        tested_pos = ev["hit"] + ev["missed"]
        train.update({
            "missed_rate": ev["missed"] / max(tested_pos, 1),
            "false_positive_rate": ev["false_positive"] / max(3 * E - tested_pos, 1),
            "detector_flags_per_step": tested_pos, "predicted_per_step": ev["predicted"],
            "timed_run": {"predicted": in_run["predicted"], "missed_caught_by_detector": in_run["missed"]}})
    # "at fixed L2 error": every run's relative density L2 difference to the plain float64 run after
    # the same K steps; the headline is the fastest run within the gate
    gate = 1e-6
    for name, r in runs.items():
        if "float64" in runs and name != "float64":
            a, b = r["U"], runs["float64"]["U"]
            num = sum(float(((a[k][..., 0] - b[k][..., 0]) ** 2).sum()) for k in a)
            den = sum(float((b[k][..., 0] ** 2).sum()) for k in b)
            r["l2"] = (num / den) ** 0.5
        else:
            r["l2"] = 0.0
    eligible = [k for k in runs if runs[k]["l2"] <= gate]
    head = max(eligible, key=lambda k: runs[k]["value"])
    head_prec = "mixed" if "mixed" in head else "float64"
    R = runs[head]
    op, (limiter, integ) = ops[head_prec], integs[head_prec]
    troubled = None
    if args.limiter == "mood":
        flags = limiter.troubled(R["U"])
        troubled = int(sum(int(v.sum().item()) for v in flags.values()))
    accuracy = {"density_l2_rel_vs_plain": {k: v["l2"] for k, v in runs.items()}, "after_steps": args.steps,
                "gate": gate, "headline": head, "within_gate": eligible}

    # per-stage kernel durations of one RHS (CUDA events on the launching stream)
    stage_ms = (ctypes.c_float * len(STAGES))()
    st = op.native.state(op._blocks(R["U"]))
    for _ in range(3):
        N.check(N.lib().dgb_rhs_profile(op.native.handle, ctypes.byref(st), stage_ms, _stream_ptr()))
    stages = dict(zip(STAGES, [float(x) for x in stage_ms]))
    fused = bool(getattr(op.native, "fused", True)) and op.native.sum_factorised
    sbytes = stage_bytes_fused(op, nv, split=True) if fused else stage_bytes(op, nv, split=True)
    dominant = max(stages, key=stages.get)
    pk, pk_kind = peaks()
    hbm = float(pk["hbm_gbs"])
    achieved = sbytes[dominant] / (stages[dominant] / 1e3) / 1e9
    traffic = None
    tfile = ROOT / "profiles" / "traffic.json"
    if tfile.exists():
        try:
            table = json.loads(tfile.read_text())
            per_elem = (table.get("fused", {}) if fused else table).get(dominant, {}).get("dram_bytes_per_element")
            if per_elem:
                traffic = per_elem * E
        except Exception:
            traffic = None

    # end to end through the public API with host buffers.  Every step is a request of its own: its
    # state goes host -> device from pinned memory, one checked step runs, the stepped state goes
    # device -> host.  The host copies run on two copy streams through device staging buffers, so the
    # upload of step k+1 and the download of step k-1 overlap the compute of step k; the step works on
    # one fixed device state (its CUDA graph stays valid), filled from and drained to the staging
    # buffers by device-to-device copies on the compute stream.  The first upload and the last
    # download are not overlapped and stay inside the timed region.
    learned_head = head.startswith("learned")
    if learned_head:
        predictor.attach("learned")
    host_in = {k: v.cpu().pin_memory() for k, v in U_start.items()}
    host_out = {k: torch.empty_like(v).pin_memory() for k, v in host_in.items()}
    dev = {k: torch.empty_like(v) for k, v in U_start.items()}
    stage_in = {k: torch.empty_like(v) for k, v in U_start.items()}
    stage_out = {k: torch.empty_like(v) for k, v in U_start.items()}
    comp = torch.cuda.current_stream()
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    in_ready, in_free, out_ready, out_free = (torch.cuda.Event() for _ in range(4))
    e_steps = max(1, args.steps)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(comp)
    up.wait_event(e0)
    with torch.cuda.stream(up):
        for k in dev:
            stage_in[k].copy_(host_in[k], non_blocking=True)
    in_ready.record(up)
    for s in range(e_steps):
        comp.wait_event(in_ready)
        for k in dev:
            dev[k].copy_(stage_in[k], non_blocking=True)
        in_free.record(comp)
        if s + 1 < e_steps:
            up.wait_event(in_free)
            with torch.cuda.stream(up):
                for k in dev:
                    stage_in[k].copy_(host_in[k], non_blocking=True)
            in_ready.record(up)
        integ.checked_step_inplace(dev, dt, bc)
        if s > 0:
            comp.wait_event(out_free)
        for k in dev:
            stage_out[k].copy_(dev[k], non_blocking=True)
        out_ready.record(comp)
        down.wait_event(out_ready)
        with torch.cuda.stream(down):
            for k in dev:
                host_out[k].copy_(stage_out[k], non_blocking=True)
        out_free.record(down)
    comp.wait_event(out_free)
    e1.record(comp)
    torch.cuda.synchronize()
    if learned_head:
        predictor.attach("off")
    e2e_ms = e0.elapsed_time(e1) / e_steps
    # the result that came back is the stepped state (compared with the device-side step)
    e2e_ok = all(torch.equal(host_out[k], dev[k].cpu()) for k in dev)
    state_bytes = sum(v.numel() * 8 for v in host_in.values())

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.cpu_seconds)
    # launches per checked step: per stage the RHS kernels (per block / face type), then the
    # limiter and admissibility kernels (and the predictor's three per block when learned)
    nb, nf = len(op.plan.blocks), len(op.plan.faces)
    if fused:
        per_stage = 2 * nb + nf                    # traces, face kernel, element kernel
    else:
        per_stage = nb * (4 if (op.native.sum_factorised and op.viscous) else 3) + nf * (2 if op.viscous else 1)
    if args.limiter == "mood":
        per_stage += nb * 6 + nf + nb + 1
        if learned_head:
            per_stage += 3 * nb
    else:
        per_stage += nb * 2 + 1
    if op.native.sum_factorised:
        # the certificate pre-pass before each positivity pass (two per stage with MOOD) and the
        # sensor pre-pass before the troubled-cell test (MOOD)
        per_stage += 3 if args.limiter == "mood" else 1
    lim = "MOOD subcell FV (CWENO-Z) + positivity" if args.limiter == "mood" else "positivity limiter"
    prec = ("mixed: float32 arithmetic in the traces, BR2-lift, volume and finalize kernels; float64 state, "
            "face fluxes, limiters and reductions" if head_prec == "mixed" else "plain float64")
    line = {
        "metric": METRIC, "value": R["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": R["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if head_prec == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": f"Mach-3 viscous sphere, O/H hex grid, {E} elements, P{args.degree} ({dofs} DOF), "
                               f"checked SSP-RK3 with {lim}, {prec}"
                               + (", learned troubled-cell predictor" if learned_head else ""),
                   "elements": E, "degree": args.degree, "dofs": int(dofs), "mode": head,
                   "start": ("Mach-3 normal-shock state in the elements inside r < 0.65, free stream outside"
                             if args.start == "shock" else "uniform free stream"),
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (state 0.5 GB, inverse mass 6.6 GB per pass)",
                   "limiter": args.limiter, "troubled_elements_after": troubled, "setup_s": round(setup_s, 1),
                   "cuda_graph_step": bool(args.graph),
                   "rhs_form": {m: f.get("chosen") for m, f in forms.items()},
                   "rhs_form_ms": {m: {k: v for k, v in f.items() if k != "chosen"} for m, f in forms.items()}},
        "gpu_launches": per_stage * 3 * args.steps,
        "step_status": {"valid": R["valid"], "rho_min": R["rho_min"], "p_min": R["p_min"], "dt": dt},
        "stage_ms": stages,
        "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_kind": pk_kind, "traffic": traffic,
                     "algorithmic_bytes": sbytes[dominant],
                     "stage_achieved_gbs": {k: sbytes[k] / (stages[k] / 1e3) / 1e9 if stages[k] > 0 else None
                                            for k in STAGES},
                     "rhs_algorithmic_bytes": rhs_bytes(op, nv),
                     "rhs_achieved_gbs": rhs_bytes(op, nv) / (sum(stages.values()) / 1e3) / 1e9},
        "clocks": R["clocks"],
        "e2e": {"value": dofs / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes, "steps": e_steps, "ms_per_step": e2e_ms,
                "result_matches_device": e2e_ok,
                "copies": "pinned host buffers; upload of step k+1 and download of step k-1 on two copy "
                          "streams overlap step k (device staging buffers); first upload and last download "
                          "not overlapped"},
        "runs": {k: {"value": v["value"], "ms_per_step": v["ms"] / args.steps, "valid": v["valid"],
                     "density_l2_rel_vs_plain": v["l2"], "clocks_sm_mhz": v["clocks"].get("sm_mhz"),
                     "reasons": v["clocks"].get("reasons")}
                 for k, v in runs.items()},
        "accuracy": accuracy,
    }
    if train:
        line["predictor"] = train
    if cpu:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


class CpuSample:
    """Oracle (numpy float64 restatement of the reference) on a bounded sample of the workload:
    a coarse sphere O/H grid at P3 from the same shocked start, whole checked SSP-RK3 steps with
    MOOD, all host threads for BLAS."""

    def __init__(self):
        from oracle.dg import Operator, PositivityLimiter, TimeIntegrator
        from oracle.mesh import Mesh, MeshSource
        from oracle.physics import FarfieldWallBoundary, Gas
        src = workload("tiny")
        u, mu, farfield = freestream(3)
        mesh = Mesh(MeshSource(src.points, src.cells, src.physical, src.field_data))
        gas = Gas(dynamic_viscosity=mu)
        op = Operator(mesh, gas, 3)
        self.bc = FarfieldWallBoundary(gas, mesh.physical_names, farfield, wall_temperature=T_WALL / T_INF)
        from oracle.subcell import MOODLimiter
        self.integ = TimeIntegrator(op, cfl=0.3, limiter=MOODLimiter(op, positivity=PositivityLimiter(op)))
        from oracle.elements import RefElement
        g, M = GAMMA, MACH
        rho2 = (g + 1) * M ** 2 / ((g - 1) * M ** 2 + 2)
        p2 = 1 + 2 * g / (g + 1) * (M ** 2 - 1)
        self.states = {}
        for b in mesh.element_blocks:
            # the same shocked start as the GPU run (bow_shock_state), at first-order node positions
            nodes = RefElement(b.element_type, 3).nodes
            xyz = np.einsum("qi,eid->eqd", RefElement(b.element_type, 1).basis(nodes), mesh.points[b.connectivity])
            inside = shock_layer(xyz)
            W = np.zeros(xyz.shape[:-1] + (5,))
            W[..., 0] = np.where(inside, rho2, 1.0)
            W[..., 1] = np.where(inside, u / rho2, u)
            W[..., 4] = np.where(inside, p2, 1.0)
            self.states[b.element_type] = gas.to_conserved(W)
        self.dt = self.integ.stable_dt(self.states)
        self.elements = sum(len(b.connectivity) for b in mesh.element_blocks)
        self.dofs = self.elements * 64

    def step(self):
        t0 = time.time()
        self.states = self.integ.checked_step(self.states, self.dt, self.bc)[0]
        return time.time() - t0


def cpu_baseline(budget_s=15.0):
    sample = CpuSample()
    steps, sec = 0, 0.0
    while steps == 0 or sec < budget_s:
        sec += sample.step()
        steps += 1
    return {"value": sample.dofs * steps / sec, "unit": UNIT, "cores": len(os.sched_getaffinity(0)),
            "kind": "port",
            "sample": f"oracle checked SSP-RK3 steps (MOOD) on a {sample.elements}-element P3 sphere O/H grid, "
                      f"{steps} steps in {sec:.1f} s, float64 numpy"}


def run_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    sample = CpuSample()
    for _ in range(args.warmup):
        sample.step()
    sec = sum(sample.step() for _ in range(args.steps))
    value = sample.dofs * args.steps / sec
    cb = {"value": value, "unit": UNIT, "cores": len(os.sched_getaffinity(0)), "kind": "port",
          "sample": f"oracle checked SSP-RK3 steps (MOOD) on a {sample.elements}-element P3 sphere O/H grid, "
                    f"{args.steps} timed steps in {sec:.1f} s, float64 numpy (the reference is Python/JAX; "
                    f"JAX is not installable here, so its numpy restatement is timed)"}
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "Mach-3 viscous sphere O/H hex grid, P3: bounded coarse sample on host cores"},
            "cpu_baseline": cb,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--scale", default="full", choices=["full", "medium", "small", "tiny"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--limiter", default="mood", choices=["mood", "positivity"])
    ap.add_argument("--graph", type=int, default=1, help="replay each checked step as one CUDA graph")
    ap.add_argument("--start", default="shock", choices=["shock", "uniform"])
    ap.add_argument("--learned", type=int, default=1, help="train and use the troubled-cell predictor (MOOD)")
    ap.add_argument("--train-steps", type=int, default=20)
    ap.add_argument("--train-epochs", type=int, default=8)
    ap.add_argument("--threshold", type=float, default=0.9,
                    help="predictor probability above which an element skips the a-posteriori test")
    ap.add_argument("--precision", default="both", choices=["both", "mixed", "float64"],
                    help="both: time the plain float64 step and the mixed step from the same state and dt; "
                         "the mixed one is the headline value, the plain one and their density L2 "
                         "difference ride along")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
