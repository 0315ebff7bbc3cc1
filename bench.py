"""Benchmark: RK-stage DOF-updates/s of the explicit DG step.

Workload (one GPU): Navier-Stokes Taylor-Green vortex, periodic [0, 2 pi]^3,
32^3 hexes, p = 3 (64 DOF per element per variable), Re 1600, Ma 0.1, BR2
viscous terms, RK4 with dt = 0.2 h / ((2p+1)(c + |u|max)), FP64.  Synthetic
initial data (the analytic TGV field), no dataset.  A "step" is one RK4 time
step = 4 RK stages; DOF-updates per stage = 5 * 64 * 32^3.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Our arm: the state stays resident in HBM; `value` is device time (CUDA events
on the handle's stream, max over ranks) of K graph-launched steps; `e2e` is the
same metric through the C ABI with host buffers (pinned H2D of the state, the
step, D2H of the state and the residual norm, every step).  Multi-GPU runs
are independent replicas (weak scaling): the reference's multi-rank mode is a
domain decomposition this library does not implement.

--impl reference: the reference's own FP64 CPU solver (compiled in place into
oracle/_ref/) on the host cores, one process per core, each step a bounded
sample of the same workload (a 6^3 block of the 32^3 TGV mesh; identical
per-element work), DOF-updates/s summed over processes.
"""
import argparse
import json
import math
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "RK-stage DOF-updates/s (FP64, TGV 32^3 p=3 RK4)"
UNIT = "DOF-updates/s"
# B200 FP64 arithmetic peak: 148 SMs x 64 FP64 FMA lanes x 2 flop x 1.965 GHz
# (nominal; the FP64 rate is not among the measured peaks)
FP64_PEAK_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12
FP64_PEAK_SOURCE = "nominal: 148 SMs x 64 FP64 FMA/clk x 2 x 1965 MHz"
N_EL = 32
P_ORD = 3
L_BOX = 2 * math.pi


def tgv_case(n, p):
    from tests import cases as C
    nodes = C.box_nodes(n, n, n, 1, L_BOX, L_BOX, L_BOX)
    prm = C.params(mu=1.0 / 1600.0, c=10.0, u=0.0, v=0.0, w=0.0)
    U = C.taylor_green(C.node_coords(n, n, n, p, 1, nodes)).reshape(-1)
    dt = 0.2 * (L_BOX / n) / ((2 * p + 1) * (10.0 + 1.0))
    return nodes, prm, U, dt


def config():
    """The workload both arms report (the same dict in both lines)."""
    return {"workload": f"Taylor-Green vortex Re=1600 Ma=0.1, periodic [0,2pi]^3, {N_EL}^3 hexes, p={P_ORD}, BR2, "
                        f"RK4, FP64",
            "nelem": N_EL ** 3, "p": P_ORD, "dof_per_stage": 5 * (P_ORD + 1) ** 3 * N_EL ** 3,
            "scheme": "RK4", "l2_between_steps": "inputs larger than L2 (trace buffer 252 MB + 3 state arrays "
                                                 "84 MB each)"}


# ------------------------------------------------------------- reference arm

def _ref_worker(args):
    """One process: the reference solver on a small block of the TGV mesh.
    Returns the stage time (s) of its RK4 step, geometry set-up excluded."""
    nsteps, n = args
    import oracle
    ref = oracle.reference()
    nodes, prm, U, dt = tgv_case(n, P_ORD)
    m = oracle.Mesh(n, n, n, P_ORD, 1, nodes, [-2] * 6)
    t0 = time.perf_counter()
    ref.run(m, prm, U, 0, dt, 0)          # geometry precompute only
    t1 = time.perf_counter()
    ref.run(m, prm, U, 0, dt, nsteps)     # precompute + nsteps RK4 steps
    t2 = time.perf_counter()
    stage_s = max((t2 - t1) - (t1 - t0), 1e-9) / (4 * nsteps)
    return stage_s


REF_BLOCK = 6  # elements per direction of one reference process's sample block


def cpu_rate(nsteps, n, procs, pool=None):
    """DOF-updates/s of `procs` concurrent reference processes (a spawn pool
    is made for the call unless one is passed in), and their stage times."""
    import multiprocessing as mp
    if pool is None:
        with mp.get_context("spawn").Pool(procs) as p:
            return cpu_rate(nsteps, n, procs, p)
    stage_s = pool.map(_ref_worker, [(nsteps, n)] * procs)
    dof = 5 * (P_ORD + 1) ** 3 * n ** 3
    return sum(dof / s for s in stage_s), stage_s


def host_cores():
    """(logical, physical) host core counts."""
    logical = os.cpu_count() or 1
    physical = None
    try:
        import psutil
        physical = psutil.cpu_count(logical=False)
    except ImportError:
        pass
    return logical, physical


def run_reference(args, rank, world):
    """The reference's own FP64 CPU solver on every host thread.  A step is
    one sample: every process runs one RK4 step of a 6^3 block of the TGV
    mesh (periodic, same p, so the same work per element), all processes at
    once.  `value` is the summed DOF-updates/s of the processes (median over
    steps); `ms_per_step` is the measured time of a sample step (the mean
    over processes of their RK4 step), not the cost of a full 32^3 step,
    which is reported beside it as an extrapolation."""
    if rank != 0:
        return
    import oracle
    if oracle.reference() is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdgref.so was not built "
                          "(the reference tree is needed to compile it)"}))
        return
    import multiprocessing as mp
    procs, physical = host_cores()
    n = REF_BLOCK
    rates, step_s = [], []
    with mp.get_context("spawn").Pool(procs) as pool:  # one pool for the run
        for i in range(args.warmup + args.steps):
            r, st = cpu_rate(1, n, procs, pool)
            if i >= args.warmup:
                rates.append(r)
                step_s.append(4 * float(np.mean(st)))
    with mp.get_context("spawn").Pool(1) as pool:  # one process alone: the per-core rate
        single, _ = cpu_rate(1, n, 1, pool)
    value = float(np.median(rates))
    dof32 = 5 * (P_ORD + 1) ** 3 * N_EL ** 3
    sample = (f"{procs} concurrent single-rank reference processes ({physical} physical cores), each one RK4 "
              f"step of a {n}^3 block (periodic, same p, same per-element work) of the {N_EL}^3 TGV per bench step; "
              f"stage time = (wall with the step - wall of geometry set-up alone) / 4")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(step_s)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": procs, "physical_cores": physical,
                         "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "ms_per_step_is": f"the measured RK4 step of one {n}^3 sample block per process (all processes at once)",
        "samples_run": {"bench_steps": args.steps, "warmup_steps": args.warmup,
                        "rk4_steps_per_process_per_bench_step": 1, "processes": procs},
        "full_step_ms_extrapolated": 4 * dof32 / value * 1e3,
        "single_process_rate": {"value": single, "unit": UNIT, "cores": 1,
                                "sample": f"one process alone, one RK4 step of a {n}^3 block"},
    }))


# ------------------------------------------------------------------ our arm

class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join("/tmp", f"dgb_clocks_{os.getpid()}_{gpu}.csv")

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.f.close()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(x, device="cuda"):
    """The maximum of a per-rank number over all ranks of the default process
    group (the rank itself when there is none): the multi-GPU time of a step
    is the slowest replica's."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return x
    t = torch.tensor([x], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, dof_stage, stages_per_step, steps, ms):
    """Whole-job DOF-updates/s of `world` independent replicas, each doing
    `steps` steps in `ms` (the max over ranks)."""
    return world * dof_stage * stages_per_step * steps / (ms * 1e-3)


def _timed_steps(dg, torch, s, stream, dt, steps, scheme=None):
    """Device time (ms) of `steps` graph-launched RK steps (default RK4) on the handle's stream."""
    scheme = dg.RK4 if scheme is None else scheme
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        s.step(scheme, dt, steps, norms=True)
        ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1)


def _warm(dg, torch, s, dt, min_steps, min_seconds=0.5, scheme=None):
    scheme = dg.RK4 if scheme is None else scheme
    t_w = time.perf_counter()
    warm = 0
    while warm < min_steps or time.perf_counter() - t_w < min_seconds:
        s.step(scheme, dt, 1, norms=False)
        warm += 1
    torch.cuda.synchronize()
    return warm


def _stage_kernel_ms(dg, s, U0, dt, reps):
    """Mean per-launch durations (CUDA events on the launching stream) of the
    stage kernel and of the trace kernel; launch order of one profiled step:
    initial traces, stage0, norm, stage1, stage2, stage3."""
    s.set_state(U0)
    kms = s.profile_step(dg.RK4, dt, reps)
    return float(np.mean([kms[1], kms[3], kms[4], kms[5]])), float(kms[0])


def _reverse_step_ms(dg, torch, s, stream, U0, dt, reps):
    """Device time (ms, CUDA events on the handle's stream) of one reverse RK4
    step (3 stage recomputations + 4 residual VJPs) at state U0."""
    Ud = torch.tensor(U0, device="cuda")
    lam = torch.ones_like(Ud)
    torch.cuda.synchronize()
    s.step_vjp_device(dg.RK4, dt, Ud.data_ptr(), lam.data_ptr())  # warm-up, allocates the adjoint buffers
    launches = s.last_launch_count
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    tot = 0.0
    for _ in range(reps):
        lam.fill_(1.0)
        torch.cuda.synchronize()
        ev0.record(stream)
        s.step_vjp_device(dg.RK4, dt, Ud.data_ptr(), lam.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        tot += ev0.elapsed_time(ev1)
    return tot / reps, launches


def _reverse_sweep_ms(dg, torch, s, stream, U0, dt, k):
    """Device time (ms, CUDA events on the handle's stream) per reverse RK4
    step inside one backward sweep over a recorded run of k steps that kept
    every state (nothing recomputed): the sweep's k state restores and its
    two adjoint basis conversions are spread over its k reverse steps, where
    the single-step call pays three conversions per step."""
    s.set_state(U0)
    s.forward_record(dg.RK4, dt, k, k, norms=False)
    lam = torch.ones(s.n, dtype=torch.float64, device="cuda")
    out = torch.empty_like(lam)
    torch.cuda.synchronize()
    s.backward_device(lam.data_ptr(), out.data_ptr())  # warm-up
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    tot = 0.0
    for _ in range(3):
        torch.cuda.synchronize()
        ev0.record(stream)
        s.backward_device(lam.data_ptr(), out.data_ptr())
        ev1.record(stream)
        torch.cuda.synchronize()
        tot += ev0.elapsed_time(ev1)
    recomputed, reversed_, _ = s.adjoint_stats()
    if recomputed != 0 or reversed_ != k:
        raise RuntimeError(f"sweep recomputed {recomputed} and reversed {reversed_} of {k} steps")
    return tot / 3 / k


def _adjoint_config(dg, torch, nsteps, budgets):
    """Gradient of the final enstrophy w.r.t. the 8 x 3 amplitudes of seeded
    Fourier velocity modes on a uniform flow: periodic [0, 2 pi]^3, 16^3 hexes,
    p = 3, Re 500, Ma 0.3, RK4, FP64.  Times the recorded forward run and the
    backward sweep for each checkpoint budget (a number of state buffers, or
    -1: every state and stage state kept), and checks the gradient along
    one random direction against central differences of two plain runs."""
    from dgpr_b200 import autograd as dga
    from dgpr_b200 import functionals as F
    from tests import cases as C
    n, p, Re, Ma = 16, 3, 500.0, 0.3
    c = 1.0 / Ma
    prm = C.params(mu=1.0 / Re, c=c, u=1.0, v=0.0, w=0.0)
    nodes = C.box_nodes(n, n, n, 1, L_BOX, L_BOX, L_BOX)
    xyz = F.box_node_coords(n, n, n, p, L_BOX, L_BOX, L_BOX)
    modes = F.FourierModes(xyz, 1.4, 1.0, prm[5], (1.0, 0.0, 0.0), nmodes=8, kmax=4, amp=0.05, seed=0,
                           device="cuda")
    quad = F.BoxQuadrature(n, n, n, p, L_BOX, L_BOX, L_BOX, device="cuda")
    dt = 0.2 * (L_BOX / n) / ((2 * p + 1) * (c + 1.5))
    mesh = dg.Mesh(n, n, n, p, 1, nodes, [dg.PERIODIC] * 6)
    out = {"workload": f"Fourier modes on uniform flow, periodic [0,2pi]^3, {n}^3 hexes, p={p}, Re={Re:g}, "
                       f"Ma={Ma:g}, RK4 dt={dt:.3e}, {nsteps} steps, J = final enstrophy, 24 amplitudes",
           "budgets": []}
    with dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64) as s:
        a0 = modes.amplitudes("cuda")
        U0 = modes.state(a0).detach()
        s.set_state(U0.cpu().numpy())
        s.step(dg.RK4, dt, 5, norms=False)  # warm-up
        # untimed backward of a short record: the reverse-step graph and the
        # adjoint buffers are made on first use, outside the timed budgets
        s.set_state(U0.cpu().numpy())
        s.forward_record(dg.RK4, dt, 2, 2, norms=False)
        s.backward(np.zeros(U0.numel()))
        grad = None
        reps = 3  # host wall clock on a small mesh: the median of three runs
        for slots in budgets:
            # untimed recorded run first: allocates (or frees) the checkpoint buffers
            s.set_state(U0.cpu().numpy())
            if slots == dga.STAGES:
                s.forward_record_stages(dg.RK4, dt, nsteps, norms=False)
            else:
                s.forward_record(dg.RK4, dt, nsteps, slots, norms=False)
            tf, tb, same = [], [], True
            for _ in range(reps):
                a = a0.clone().requires_grad_(True)
                Ua = modes.state(a)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                UN = dga.integrate(Ua, s, dg.RK4, dt, nsteps, slots=slots)
                torch.cuda.synchronize()
                t1 = time.perf_counter()
                J = F.enstrophy(UN, quad)
                J.backward()
                torch.cuda.synchronize()
                t2 = time.perf_counter()
                tf.append(t1 - t0)
                tb.append(t2 - t1)
                fwd, rev, planned = s.adjoint_stats()
                g = a.grad.cpu().numpy()
                if grad is None:
                    grad = g
                same = same and bool(np.array_equal(g, grad))
            out["budgets"].append({"slots": "every state and stage state" if slots == dga.STAGES else slots,
                                   "recorded_forward_s": float(np.median(tf)), "backward_s": float(np.median(tb)),
                                   "runs": reps, "recomputed_steps": fwd, "reversed_steps": rev,
                                   "gradient_equal_to_first_budget": same})
        # plain forward time of the same run (no recording), median of three
        tp = []
        for _ in range(reps):
            s.set_state(U0.cpu().numpy())
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.step(dg.RK4, dt, nsteps, norms=False)
            torch.cuda.synchronize()
            tp.append(time.perf_counter() - t0)
        out["plain_forward_s"] = float(np.median(tp))
        for b in out["budgets"]:
            b["backward_over_plain_forward"] = b["backward_s"] / out["plain_forward_s"]
        rng = np.random.default_rng(1)
        d = torch.tensor(rng.standard_normal((8, 3)), device="cuda")

        def Jof(av):
            s.set_state(modes.state(av).detach().cpu().numpy())
            s.step(dg.RK4, dt, nsteps, norms=False)
            return float(F.enstrophy(torch.tensor(s.get_state(), device="cuda"), quad))

        h = 1e-5
        fd = (Jof(a0 + h * d) - Jof(a0 - h * d)) / (2 * h)
        an = float((torch.tensor(grad, device="cuda") * d).sum())
        out["fd_check"] = {"directional_adjoint": an, "directional_fd": fd, "rel_err": abs(an - fd) / abs(fd),
                           "h": h}
        # every one of the 24 components by central differences of FP64 forward
        # runs, h = 1e-4 |a_k|; the error is taken against the gradient's
        # largest component
        a0h = a0.detach().cpu().numpy().ravel()
        fdv = np.zeros(a0h.size)
        for k in range(a0h.size):
            hk = 1e-4 * max(abs(a0h[k]), 1e-3)
            e = torch.zeros_like(a0).view(-1)
            e[k] = hk
            e = e.view_as(a0)
            fdv[k] = (Jof(a0 + e) - Jof(a0 - e)) / (2 * hk)
        gv = np.asarray(grad).ravel()
        out["fd_full"] = {"components": int(a0h.size), "h": "1e-4 |a_k|",
                          "max_abs_err_over_max_grad": float(np.max(np.abs(gv - fdv)) / np.max(np.abs(gv))),
                          "rel_l2": float(np.linalg.norm(gv - fdv) / np.linalg.norm(gv))}
        # the same sweep with dJ/d[mu, source] (dgb_backward_params), stage-keeping record
        s.set_state(U0.cpu().numpy())
        s.forward_record_stages(dg.RK4, dt, nsteps, norms=False)
        UN = torch.tensor(s.get_state(), device="cuda", requires_grad=True)
        F.enstrophy(UN, quad).backward()
        lamN = UN.grad.cpu().numpy()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, dpar = s.backward_params(lamN)
        tp = time.perf_counter() - t0
        t0 = time.perf_counter()
        s.backward(lamN)
        tb = time.perf_counter() - t0
        out["param_gradient"] = {"dJ_dmu": float(dpar[0]), "backward_params_s": tp, "backward_s": tb,
                                 "over_backward": tp / tb}
    return out


def _curved_block(dg, torch, steps):
    """The same TGV workload on curved elements: the 32^3 box sinusoidally
    mapped (q = 2 nodes, y displaced by 0.1 sin x sin z), so every element
    carries per-point geometry.  Device time per step of both forms."""
    from tests import cases as C
    n, p, q = N_EL, P_ORD, 2
    nodes = C.sine_nodes(n, n, n, q, L_BOX, L_BOX, L_BOX, 0.1)
    prm = C.params(mu=1.0 / 1600.0, c=10.0, u=0.0, v=0.0, w=0.0)
    U0 = C.taylor_green(C.node_coords(n, n, n, p, q, nodes)).reshape(-1)
    dt = 0.2 * (L_BOX / n) / ((2 * p + 1) * (10.0 + 1.0))
    mesh = dg.Mesh(n, n, n, p, q, nodes, [dg.PERIODIC] * 6)
    stream = torch.cuda.Stream()
    out = {"workload": f"TGV on a sinusoidally mapped {n}^3 mesh, q = {q}, p = {p}, RK4 (per-point geometry)"}
    for prec, name in ((dg.FP64, "fp64"), (dg.MIXED_FP32, "mixed")):
        with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
            s.set_stream(stream.cuda_stream)
            s.set_state(U0)
            _warm(dg, torch, s, dt, 3)
            ms = _timed_steps(dg, torch, s, stream, dt, steps) / steps
        out[name] = {"ms_per_step": ms, "value": 5 * (p + 1) ** 3 * n ** 3 * 4 / (ms * 1e-3), "unit": UNIT}
    return out


def _heat_block(dg, torch, steps):
    """The headline workload with the configuration's Pr = 0.71 heat flux
    (dgb_set_prandtl; the reference has no heat conduction, so this is not
    comparable to its arm).  Device time per step of both forms."""
    nodes, prm, U0, dt = tgv_case(N_EL, P_ORD)
    mesh = dg.Mesh(N_EL, N_EL, N_EL, P_ORD, 1, nodes, [dg.PERIODIC] * 6)
    stream = torch.cuda.Stream()
    out = {"workload": f"TGV {N_EL}^3 p = {P_ORD} RK4 with heat conduction, Pr = 0.71"}
    for prec, name in ((dg.FP64, "fp64"), (dg.MIXED_FP32, "mixed")):
        with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
            s.set_stream(stream.cuda_stream)
            s.set_prandtl(0.71)
            s.set_state(U0)
            _warm(dg, torch, s, dt, 3)
            ms = _timed_steps(dg, torch, s, stream, dt, steps) / steps
        out[name] = {"ms_per_step": ms, "value": 5 * (P_ORD + 1) ** 3 * N_EL ** 3 * 4 / (ms * 1e-3), "unit": UNIT}
    return out


def _channel_block(dg, torch, steps):
    """Config 5's channel: [0,4 pi] x [0,2] x [0,2 pi], 64 x 32 x 32 hexes,
    p = 3, q = 2 nodes sinusoidally mapped (y displaced by 0.1 sin(x/2) sin z,
    damped to flat walls), periodic x/z, isothermal walls in y at the
    reference temperature, Pr 0.71, body force fx for Re_tau ~ 180 (bulk Re
    5600, Ma 0.2), seeded perturbations of a parabolic profile, TVD-RK3 with
    dt from CFL 0.2.  Device time per step of both forms.  The isothermal wall
    and the heat flux are extensions (no reference counterpart)."""
    mesh, prm, U0, dt = _channel_case(dg)
    nx, ny, nz, p, q = mesh.nx, mesh.ny, mesh.nz, mesh.p, mesh.q
    stream = torch.cuda.Stream()
    out = {"workload": f"channel {nx}x{ny}x{nz} hexes, p = {p}, q = {q} sinusoidal map, isothermal walls, Pr 0.71, "
                       f"body force, TVD-RK3 dt={dt:.3e} (CFL 0.2)"}
    for prec, name in ((dg.FP64, "fp64"), (dg.MIXED_FP32, "mixed")):
        with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
            s.set_stream(stream.cuda_stream)
            s.set_prandtl(0.71)
            s.set_state(U0)
            _warm(dg, torch, s, dt, 3, scheme=dg.TVDRK3)
            ms = _timed_steps(dg, torch, s, stream, dt, steps, scheme=dg.TVDRK3) / steps
        out[name] = {"ms_per_step": ms, "value": 5 * (p + 1) ** 3 * nx * ny * nz * 3 / (ms * 1e-3), "unit": UNIT}
    return out


def _channel_case(dg):
    from tests import cases as C
    nx, ny, nz, p, q = 64, 32, 32, P_ORD, 2
    lx, ly, lz = 4 * math.pi, 2.0, 2 * math.pi
    nu = ly / 5600.0
    utau = 180.0 * nu / (ly / 2)
    c = 5.0
    prm = C.params(mu=nu, c=c, u=0.0, v=0.0, w=0.0, source=(0.0, utau * utau / (ly / 2), 0.0, 0.0, 0.0))
    nodes = C.sine_nodes(nx, ny, nz, q, lx, ly, lz, 0.1, walls=True)
    xyz = C.node_coords(nx, ny, nz, p, q, nodes)
    rng = np.random.default_rng(5)
    y = xyz[..., 1]
    u = 1.5 * (1.0 - (y - 1.0) ** 2) * (1.0 + 0.05 * rng.standard_normal(y.shape))
    vv = 0.05 * rng.standard_normal(y.shape) * (1.0 - (y - 1.0) ** 2)
    U0 = C.state_from_primitives(1.0 + 0 * y, u, vv, 0 * y, prm[5] + 0 * y, prm[0]).reshape(-1)
    dt = 0.2 * (ly / ny) / ((2 * p + 1) * (c + 1.5))
    iso = dg.ISOTHERMAL_WALL
    mesh = dg.Mesh(nx, ny, nz, p, q, nodes, [dg.PERIODIC, dg.PERIODIC, iso, iso, dg.PERIODIC, dg.PERIODIC])
    return mesh, prm, U0, dt


def _channel_adjoint_block(dg, torch, nsteps, slots=50):
    """The adjoint-at-scale configuration on config 5's channel: `nsteps`
    TVD-RK3 steps recorded with `slots` checkpoint buffers, then the FP64
    adjoint sweep giving dJ/dT_w for J = the mean wall shear stress of the
    y = 0 wall at the end (functionals.wall_shear, with the box metric of the
    unmapped mesh; the sinusoidal map leaves the walls flat).  Two gradients:
    the configuration's (mixed-form forward record: FP32 contractions and
    fluxes, FP64 adjoint) and the all-FP64 one.  The reference value is
    central differences of FP64 forward runs at two steps, h = 1e-4 T_w and
    h/2, Richardson-extrapolated, so the differencing error is not charged to
    either gradient: the FP64 gradient's error against it is the adjoint's,
    and the mixed gradient's distance from the FP64 gradient is the cost of
    the mixed forward.  The isothermal wall, the heat flux and this gradient
    have no reference counterpart."""
    from dgpr_b200 import functionals as F
    mesh, prm, U0, dt = _channel_case(dg)
    lx, ly, lz = 4 * math.pi, 2.0, 2 * math.pi
    quad = F.BoxQuadrature(mesh.nx, mesh.ny, mesh.nz, mesh.p, lx, ly, lz, device="cuda")
    mu, Tw = prm[2], prm[4]

    def J_of(U):
        return F.wall_shear(U, quad, mu, wall="-y")

    out = {"workload": f"channel {mesh.nx}x{mesh.ny}x{mesh.nz} p = {mesh.p} q = {mesh.q}, isothermal walls at "
                       f"T_w = {Tw:.4g}, Pr 0.71, {nsteps} TVD-RK3 steps dt={dt:.3e}; J = mean wall shear of "
                       f"the y = 0 wall; FP64 adjoint, {slots} checkpoint slots; forward record mixed (the "
                       f"configuration) and FP64"}
    grads = {}
    for prec, name in ((dg.MIXED_FP32, "mixed_forward"), (dg.FP64, "fp64_forward")):
        with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
            s.set_prandtl(0.71)
            s.set_state(U0)
            s.step(dg.TVDRK3, dt, 3, norms=False)  # warm-up
            s.set_state(U0)
            s.forward_record(dg.TVDRK3, dt, 2, 2, norms=False)
            s.backward(np.zeros(U0.size))  # warm-up of the sweep
            s.set_state(U0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s.step(dg.TVDRK3, dt, nsteps, norms=False)
            torch.cuda.synchronize()
            plain = time.perf_counter() - t0
            s.set_state(U0)
            t0 = time.perf_counter()
            s.forward_record(dg.TVDRK3, dt, nsteps, slots, norms=False)
            torch.cuda.synchronize()
            rec = time.perf_counter() - t0
            UN = torch.tensor(s.get_state(), device="cuda", requires_grad=True)
            J = J_of(UN)
            J.backward()
            lamN = UN.grad.cpu().numpy()
            t0 = time.perf_counter()
            _, dp = s.backward_params(lamN)
            back = time.perf_counter() - t0
            fwd, rev, _ = s.adjoint_stats()
        grads[name] = float(dp[dg.DPARAM_TWALL])
        out[name] = {"J": float(J.detach()), "dJ_dTw": grads[name], "plain_forward_s": plain,
                     "recorded_forward_s": rec, "backward_s": back, "backward_over_plain_forward": back / plain,
                     "recomputed_steps": fwd, "reversed_steps": rev}
    fd = {}
    with dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64) as s:
        s.set_prandtl(0.71)
        for k, h in (("h", 1e-4 * Tw), ("h/2", 0.5e-4 * Tw)):
            Js = []
            for t in (Tw + h, Tw - h):
                s.set_wall_temperature(t)
                s.set_state(U0)
                s.step(dg.TVDRK3, dt, nsteps, norms=False)
                Js.append(float(J_of(_device_state(s, torch))))
            fd[k] = (Js[0] - Js[1]) / (2 * h)
    rich = (4 * fd["h/2"] - fd["h"]) / 3
    out["fd_fp64"] = {"h": 1e-4 * Tw, "central_h": fd["h"], "central_h2": fd["h/2"], "richardson": rich,
                      "h_vs_h2_rel": abs(fd["h"] - fd["h/2"]) / abs(rich)}
    out["rel_err_fp64_adjoint_vs_fd"] = abs(grads["fp64_forward"] - rich) / abs(rich)
    out["rel_err_mixed_forward_vs_fd"] = abs(grads["mixed_forward"] - rich) / abs(rich)
    out["rel_gap_mixed_vs_fp64_adjoint"] = abs(grads["mixed_forward"] - grads["fp64_forward"]) / abs(
        grads["fp64_forward"])
    return out


def _checkpoint_block(dg, steps=600, chkints=(30, 150)):
    """Checkpoint cadence of the dgb driver (C++ host code over the C ABI,
    the drop-in for the reference's cudg): the wall time of its stepping
    loop (`-timing`: the steps and every checkpoint file, not the set-up or
    the final file) for `steps` RK4 steps of the TGV workload read from a
    .dg file, writing a .dg checkpoint every `chkint` steps, against the
    same loop with none.  The driver writes each checkpoint from a device
    snapshot on a host thread while the steps go on, so a checkpoint costs
    only what its file write exceeds the steps until the next one; with
    -chksync it writes each file before the next step, as the reference's
    cudg does, for comparison."""
    import re
    import tempfile
    exe = os.path.join(ROOT, "dgpr_b200", "_lib", "dgb")
    if not os.path.exists(exe):
        return {"unavailable": "dgpr_b200/_lib/dgb was not built"}
    nodes, prm, U0, dt = tgv_case(N_EL, P_ORD)
    mesh = dg.Mesh(N_EL, N_EL, N_EL, P_ORD, 1, nodes, [dg.PERIODIC] * 6)
    out = {"workload": f"dgb -ifile (TGV {N_EL}^3 p={P_ORD}) -scheme RK4 -niter {steps}, FP64",
           "checkpoint_bytes": int(U0.size * 8)}
    with tempfile.TemporaryDirectory() as d:
        dg.write_state(os.path.join(d, "tgv.dg"), 0, mesh, {"state": U0})
        args = [exe, "-ifile", os.path.join(d, "tgv"), "-niter", str(steps), "-scheme", "RK4", "-dt", repr(dt),
                "-mu", repr(1.0 / 1600.0), "-c", "10", "-u", "0", "-v", "0", "-w", "0", "-timing",
                "-ofile", os.path.join(d, "out")]
        runs = [("no_checkpoints_s", 10 * steps, [])] + \
               [(f"checkpoint_every_{c}_s", c, []) for c in chkints] + \
               [(f"checkpoint_every_{c}_written_before_the_next_step_s", c, ["-chksync"]) for c in chkints] + \
               [("no_checkpoints_again_s", 10 * steps, [])]
        for name, ci, extra in runs:
            r = subprocess.run(args + extra + ["-chkint", str(ci)], stdout=subprocess.DEVNULL, stderr=subprocess.PIPE,
                               check=True, timeout=600)
            m = re.search(r"steps in ([0-9.]+) s", r.stderr.decode())
            out[name] = float(m.group(1)) if m else None
    if all(out[n] for n, _, _ in runs):
        base = min(out["no_checkpoints_s"], out["no_checkpoints_again_s"])
        for c in chkints:
            out[f"overhead_frac_every_{c}"] = out[f"checkpoint_every_{c}_s"] / base - 1.0
            out[f"overhead_frac_every_{c}_written_before_the_next_step"] = \
                out[f"checkpoint_every_{c}_written_before_the_next_step_s"] / base - 1.0
            out[f"checkpoints_written_every_{c}"] = steps // c
    return out


def _reference_cuda_block(nx=16, ny=16, nz=16, k1=10, k2=2010, ours_steps=2000):
    """The reference's own GPU path, solver/cudg.cu built unmodified for
    sm_100a into oracle/_ref/cudg (FP32, thread-per-quadrature-point kernels
    with a device synchronisation after each), beside this library on the
    same workload: the reference's bump channel, nx x ny x nz hexes, p = 3,
    q = 2, turbulent initial state, subsonic inflow/outflow, inviscid walls,
    RK4 dt 1e-4.  (On an all-periodic mesh the reference's driver stops in
    its norm reduction, so the TGV box is not used here.)  Information only,
    not a parity target: the reference's CUDA path approximates BR2 by a
    local penalty and uses dt/2 in stage 3 of RK4.

    The reference is timed by the wall times of two whole driver runs,
    (k2 - k1) steps / (t(k2) - t(k1)), which removes process start and its
    set-up (its geometry precompute runs on one host core); k2 - k1 is sized
    so the difference is many seconds (process start alone varies by a
    second or two).  This library is timed in process on the same initial
    state (written by dgb -niter 0) through the C ABI call the dgb driver
    makes, `ours_steps` steps with the printed norm of every step: wall time
    (host overheads included, as in the reference's figure) and CUDA
    events."""
    import tempfile
    ref = os.path.join(ROOT, "oracle", "_ref", "cudg")
    ours = os.path.join(ROOT, "dgpr_b200", "_lib", "dgb")
    out = {"workload": f"bump channel {nx}x{ny}x{nz}, p = 3, q = 2, -turb, subsonic inflow/outflow, inviscid "
                       f"walls, RK4 dt 1e-4"}
    dof_step = 4 * 5 * 64 * nx * ny * nz
    args = ["-p", "3", "-nx", str(nx), "-ny", str(ny), "-nz", str(nz), "-turb", "-scheme", "RK4", "-dt", "1e-4",
            "-chkint", "100000000"]
    with tempfile.TemporaryDirectory() as d:
        if os.path.exists(ref):
            walls, rc = [], 0
            for k in (k1, k2):
                t0 = time.perf_counter()
                r = subprocess.run([ref] + args + ["-niter", str(k), "-ofile", os.path.join(d, f"ref{k}")],
                                   stdout=subprocess.DEVNULL, stderr=subprocess.PIPE, timeout=1200)
                walls.append(time.perf_counter() - t0)
                rc = rc or r.returncode
            if rc == 0:
                ms = 1e3 * (walls[1] - walls[0]) / (k2 - k1)
                out["reference_cudg_fp32"] = {"steps": [k1, k2], "wall_s": walls, "ms_per_step": ms,
                                              "value": dof_step / (ms * 1e-3), "unit": UNIT}
            else:
                out["reference_cudg_fp32"] = {"unavailable": f"exited {rc}: {r.stderr.decode()[-200:]}"}
        else:
            out["reference_cudg_fp32"] = {"unavailable": "oracle/_ref/cudg was not built"}
        if os.path.exists(ours):
            import dgpr_b200 as dg
            import torch
            subprocess.run([ours] + args + ["-niter", "0", "-ofile", os.path.join(d, "init")],
                           stdout=subprocess.DEVNULL, check=True, timeout=300)
            _, mesh, U = dg.read_state(os.path.join(d, "init.dg"))
            stream = torch.cuda.Stream()
            for prec, name in ((dg.FP64, "dgb_fp64"), (dg.MIXED_FP32, "dgb_mixed")):
                with dg.Solver(mesh, dg.make_reference_state(), prec) as s:
                    s.set_stream(stream.cuda_stream)
                    s.set_state(U)
                    _warm(dg, torch, s, 1e-4, 3, min_seconds=0.2)
                    torch.cuda.synchronize()
                    t0 = time.perf_counter()
                    ev_ms = _timed_steps(dg, torch, s, stream, 1e-4, ours_steps)
                    wall_ms = 1e3 * (time.perf_counter() - t0) / ours_steps
                out[name] = {"steps": ours_steps, "ms_per_step": wall_ms, "value": dof_step / (wall_ms * 1e-3),
                             "unit": UNIT, "device_ms_per_step": ev_ms / ours_steps}
    r = out.get("reference_cudg_fp32", {})
    for name in ("dgb_fp64", "dgb_mixed"):
        o = out.get(name, {})
        if "value" in r and "value" in o:
            out[f"{name}_over_reference_cuda"] = o["value"] / r["value"]
    return out


def _cpu_config_worker(name):
    """One process, one core: the reference's FP64 CPU solver on a sample of
    one benchmark configuration; returns (RK-stage DOF-updates/s, sample)."""
    import oracle
    from tests import cases as C
    ref = oracle.reference()
    if name == "config1":  # the isentropic vortex in full: 8^3, p = 2, RK4 dt 0.01
        c = [k for k in C.long_run_cases() if k.name == "vortex_8_p2_100"][0]
        m = oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
        prm, U, scheme, dt, nst, steps = c.prm, c.U, 0, c.dt, 4, 2
        sample = "the whole 8^3 p=2 vortex mesh, 2 RK4 steps"
    elif name == "config4":  # Fourier modes on a uniform flow, Re 500 Ma 0.3, p = 3
        import torch
        from dgpr_b200 import functionals as F
        n, p = 6, 3
        L = 2 * math.pi
        prm = C.params(mu=1.0 / 500.0, c=1.0 / 0.3, u=1.0, v=0.0, w=0.0)
        nodes = C.box_nodes(n, n, n, 1, L, L, L)
        xyz = F.box_node_coords(n, n, n, p, L, L, L)
        modes = F.FourierModes(xyz, 1.4, 1.0, prm[5], (1.0, 0.0, 0.0), nmodes=8, kmax=4, amp=0.05, seed=0)
        U = modes.state(modes.amplitudes("cpu")).detach().numpy().ravel()
        m = oracle.Mesh(n, n, n, p, 1, nodes, [-2] * 6)
        scheme, dt, nst, steps = 0, 0.2 * (L / 16) / (7 * (1 / 0.3 + 1.5)), 4, 1
        sample = "a periodic 6^3 block of the 16^3 configuration's flow (same p, same per-element work), 1 RK4 step"
    else:  # config 5: curved channel, q = 2, no-slip walls (the reference's), p = 3, TVD-RK3
        nx, ny, nz, p, q = 8, 4, 4, 3, 2
        lx, ly, lz = 4 * math.pi * nx / 64, 2.0 * ny / 32, 2 * math.pi * nz / 32
        nodes = C.sine_nodes(nx, ny, nz, q, lx, ly, lz, 0.1, walls=True)
        prm = C.params(mu=2.0 / 5600.0, c=5.0, u=0.0)
        rng = np.random.default_rng(5)
        U = C.random_state(prm, nx * ny * nz, (p + 1) ** 3, rng, amp=0.02).ravel()
        m = oracle.Mesh(nx, ny, nz, p, q, nodes, [-2, -2, -7, -7, -2, -2])
        scheme, dt, nst, steps = 1, 1e-4, 3, 1
        sample = "an 8x4x4 block of the channel (q = 2 sinusoidal map, the reference's no-slip walls), 1 TVD-RK3 step"
    t0 = time.perf_counter()
    ref.run(m, prm, U, scheme, dt, 0)
    t1 = time.perf_counter()
    ref.run(m, prm, U, scheme, dt, steps)
    t2 = time.perf_counter()
    stage_s = max((t2 - t1) - (t1 - t0), 1e-9) / (nst * steps)
    dof = 5 * (m.p + 1) ** 3 * m.nelem
    return dof / stage_s, sample


def _cpu_configs_block():
    """The reference's FP64 CPU solver on samples of configurations 1, 4 and
    5, one process per configuration, one core each (the reference has no
    threads): its single-core RK-stage DOF-updates/s per configuration.
    Configuration 3 (48^3, p = 4) is out of the reference's reach here: its
    geometry precompute needs more host memory than the machine has."""
    import oracle
    if oracle.reference() is None:
        return {"unavailable": "oracle/_ref/libdgref.so was not built"}
    import multiprocessing as mp
    names = ("config1", "config4", "config5")
    with mp.get_context("spawn").Pool(len(names)) as pool:
        res = pool.map(_cpu_config_worker, names)
    return {n: {"value": v, "unit": UNIT, "cores": 1, "kind": "reference", "sample": smp}
            for n, (v, smp) in zip(names, res)}


def _hbm_peak():
    """(peak GB/s, its source): the measured copy bandwidth when present."""
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (measured)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback 6650 GB/s"


def _device_state(s, torch):
    """The handle's nodal state as a CUDA float64 tensor (device-to-device)."""
    U = torch.empty(s.n, dtype=torch.float64, device="cuda")
    s.get_state_device(U.data_ptr())
    torch.cuda.synchronize()
    return U


def _config3_block(dg, torch, steps, acc_steps, ke_every=100):
    """The mixed-precision configuration's size: TGV Re 1600 Ma 0.1 on 48^3
    hexes, p = 4 (125 DOF per element and variable), RK4, dt from CFL 0.2.
    Device time per step of both forms, each form's stage-kernel roofline
    fraction (algorithmic bytes 200 nb + 80 per element and launch), and, over
    `acc_steps` steps, the relative L2 distance of the mixed state from the
    FP64 form's, with both kinetic-energy histories (every `ke_every` steps)
    and the dissipation rates -dKE/dt between them."""
    from dgpr_b200 import functionals as F
    n, p = 48, 4
    nodes, prm, U0, dt = tgv_case(n, p)
    mesh = dg.Mesh(n, n, n, p, 1, nodes, [dg.PERIODIC] * 6)
    nb = (p + 1) ** 3
    dof_stage = 5 * nb * n ** 3
    alg = (200 * nb + 80) * n ** 3
    peak, peak_src = _hbm_peak()
    stream = torch.cuda.Stream()
    out = {"workload": f"TGV Re 1600 Ma 0.1, periodic [0,2pi]^3, {n}^3 hexes, p = {p}, RK4 dt={dt:.4e}",
           "dof_per_stage": dof_stage, "algorithmic_bytes_per_stage_launch": alg, "peak_gbs": peak,
           "peak_source": peak_src}
    for prec, name in ((dg.FP64, "fp64"), (dg.MIXED_FP32, "mixed"), (dg.MIXED_FP32, "mixed_tensor_core")):
        with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
            s.set_stream(stream.cuda_stream)
            if name == "mixed_tensor_core":
                s.set_step_form(dg.STEP_GAUSS_TC)
            s.set_state(U0)
            _warm(dg, torch, s, dt, 3)
            ms = _timed_steps(dg, torch, s, stream, dt, steps) / steps
            kms, tms = _stage_kernel_ms(dg, s, U0, dt, 5)
        out[name] = {"ms_per_step": ms, "value": dof_stage * 4 / (ms * 1e-3), "unit": UNIT,
                     "stage_kernel_ms": kms, "trace_kernel_ms": tms,
                     "stage_roofline_frac": alg / (kms * 1e-3) / 1e9 / peak}
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["speedup_mixed_tensor_core_vs_fp64"] = out["mixed_tensor_core"]["value"] / out["fp64"]["value"]
    if acc_steps > 0:
        L = 2 * math.pi
        quad = F.BoxQuadrature(n, n, n, p, L, L, L, device="cuda")
        fin, ke = {}, {}
        for prec in (dg.FP64, dg.MIXED_FP32):
            with dg.Solver(mesh, dg.Params.from_array(prm), prec) as s:
                s.set_state(U0)
                hist = [float(F.kinetic_energy(_device_state(s, torch), quad))]
                done = 0
                while done < acc_steps:
                    k = min(ke_every, acc_steps - done)
                    s.step(dg.RK4, dt, k, norms=False)
                    done += k
                    hist.append(float(F.kinetic_energy(_device_state(s, torch), quad)))
                fin[prec] = _device_state(s, torch)
                ke[prec] = np.array(hist)
        err = float(torch.linalg.norm(fin[dg.MIXED_FP32] - fin[dg.FP64]) / torch.linalg.norm(fin[dg.FP64]))
        t = dt * np.minimum(np.arange(len(ke[dg.FP64])) * ke_every, acc_steps)
        eps = {k: -np.diff(v) / np.diff(t) for k, v in ke.items()}
        out["accuracy"] = {
            "steps": acc_steps, "rel_l2_mixed_vs_fp64": err, "bound": 1e-6, "within_bound": err <= 1e-6,
            "ke_every_steps": ke_every, "t": t.tolist(), "ke_fp64": ke[dg.FP64].tolist(),
            "ke_mixed": ke[dg.MIXED_FP32].tolist(),
            "dissipation_fp64": eps[dg.FP64].tolist(), "dissipation_mixed": eps[dg.MIXED_FP32].tolist(),
            "max_rel_ke_diff": float(np.max(np.abs(ke[dg.MIXED_FP32] - ke[dg.FP64]) / np.abs(ke[dg.FP64]))),
            "max_rel_dissipation_diff": float(np.max(np.abs(eps[dg.MIXED_FP32] - eps[dg.FP64])) /
                                              np.max(np.abs(eps[dg.FP64])))}
    return out


def _geometry_block(dg, torch, reps=3):
    """Set-up cost: wall time of dgb_create (allocations included), and of
    the element geometry it builds on the device (geometry.cu;
    dgb_geometry_stats), beside the host builder on the same mesh
    (dgb_geometry_host, all host threads up to 64; it excludes the
    host-to-device copy of its output that a host-built handle also needs).
    Curved: the channel mesh (per-point geometry); affine: the 48^3 p = 4
    TGV box (one Jacobian per element plus the affinity check at every
    volume point).  Median of `reps`."""
    from tests import cases as C
    mesh_c, prm_c, _, _ = _channel_case(dg)
    n3 = 48
    mesh_a = dg.Mesh(n3, n3, n3, 4, 1, C.box_nodes(n3, n3, n3, 1, L_BOX, L_BOX, L_BOX), [dg.PERIODIC] * 6)
    out = {"host_threads": min(64, os.cpu_count() or 1)}
    for name, mesh, prm in (("channel_curved", mesh_c, prm_c), ("tgv48_p4_affine", mesh_a, C.params())):
        create, build, host = [], [], []
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s = dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64)
            torch.cuda.synchronize()
            create.append(time.perf_counter() - t0)
            build.append(s.geometry_stats()[1])
            s.close()
            t0 = time.perf_counter()
            dg.geometry_host(mesh, curved=mesh.q > 1)
            host.append(time.perf_counter() - t0)
        E = mesh.nx * mesh.ny * mesh.nz
        out[name] = {"elements": E, "p": mesh.p, "q": mesh.q, "create_s": float(np.median(create)),
                     "device_geometry_build_s": float(np.median(build)), "host_builder_s": float(np.median(host))}
    return out


def run_reverse_steps(args):
    """Warm-up plus `steps` reverse RK4 steps of the FP64 adjoint at the
    workload's state (a short, profilable run of the adjoint kernels)."""
    import torch
    import dgpr_b200 as dg
    nodes, prm, U0, dt = tgv_case(N_EL, P_ORD)
    mesh = dg.Mesh(N_EL, N_EL, N_EL, P_ORD, 1, nodes, [dg.PERIODIC] * 6)
    stream = torch.cuda.Stream()
    with dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64) as s:
        s.set_stream(stream.cuda_stream)
        s.set_state(U0)
        fwd = _timed_steps(dg, torch, s, stream, dt, args.steps) / args.steps
        rev, launches = _reverse_step_ms(dg, torch, s, stream, U0, dt, args.steps)
    print(json.dumps({"workload": config()["workload"], "forward_step_ms": fwd,
                      "reverse_step_ms": rev, "reverse_over_forward": rev / fwd, "launches": launches}))


def run_ours(args, rank, world, local_rank):
    import torch
    import dgpr_b200 as dg

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
    nodes, prm, U0, dt = tgv_case(N_EL, P_ORD)
    mesh = dg.Mesh(N_EL, N_EL, N_EL, P_ORD, 1, nodes, [dg.PERIODIC] * 6)
    stream = torch.cuda.Stream()
    dof_stage = 5 * (P_ORD + 1) ** 3 * N_EL ** 3
    nb = (P_ORD + 1) ** 3

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- FP64 form: warm-up (>= W steps and >= 0.5 s, clocks sampled from
    # here), then K graph-launched steps with the state resident in HBM
    s = dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64)
    s.set_stream(stream.cuda_stream)
    s.set_state(U0)
    clk = Clocks(local_rank)
    clk.start()
    warm_run = _warm(dg, torch, s, dt, args.warmup)
    barrier()
    torch.cuda.synchronize()
    ms = max_over_ranks(_timed_steps(dg, torch, s, stream, dt, args.steps))
    barrier()
    clocks = clk.stop()
    launches = s.last_launch_count
    value = replica_rate(world, dof_stage, 4, args.steps, ms)

    # ---- end to end through the C ABI with host buffers: every step copies the
    # state in from pinned host memory and the state and norm back out
    # (dgb_step_host_async call after call on the host state in place, each
    # call's copies overlapped with its work and with the previous call's
    # copies out; dgb_synchronize at the end, inside the timed region)
    Uh = torch.empty(U0.size, dtype=torch.float64).pin_memory()
    Uh.numpy()[:] = U0
    Uhost = Uh.numpy()
    norms_h = torch.empty(1, dtype=torch.float64).pin_memory().numpy()
    for _ in range(args.warmup):  # untimed: the call's buffers, streams and piece plan are made on first use
        dg._check(dg.lib().dgb_step_host_async(s.h, dg.RK4, dt, 1, dg._p(Uhost), dg._p(Uhost), dg._p(norms_h)))
    dg._check(dg.lib().dgb_synchronize(s.h))
    Uhost[:] = U0
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dg._check(dg.lib().dgb_step_host_async(s.h, dg.RK4, dt, 1, dg._p(Uhost), dg._p(Uhost), dg._p(norms_h)))
    dg._check(dg.lib().dgb_synchronize(s.h))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e = replica_rate(world, dof_stage, 4, args.steps, e2e_s * 1e3)
    # the same with the synchronous call (each call returns with its state out)
    s.set_state(U0)
    Uhost[:] = U0
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dg._check(dg.lib().dgb_step_host(s.h, dg.RK4, dt, 1, dg._p(Uhost), dg._p(Uhost), dg._p(norms_h)))
    torch.cuda.synchronize()
    e2e_sync = replica_rate(world, dof_stage, 4, args.steps, max_over_ranks(time.perf_counter() - t0) * 1e3)
    # the same through the three plain calls (set, step, get), for comparison
    s.set_state(U0)
    Uhost[:] = U0
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        s.set_state(Uhost)
        dg._check(dg.lib().dgb_step(s.h, dg.RK4, dt, 1, dg._p(norms_h)))
        dg._check(dg.lib().dgb_get_state(s.h, dg._p(Uhost)))
    torch.cuda.synchronize()
    e2e_plain = replica_rate(world, dof_stage, 4, args.steps, max_over_ranks(time.perf_counter() - t0) * 1e3)

    reps = max(3, min(args.steps, 10))
    stage_ms, trace_ms = _stage_kernel_ms(dg, s, U0, dt, reps)
    s.close()

    # ---- mixed form, same workload
    sm = dg.Solver(mesh, dg.Params.from_array(prm), dg.MIXED_FP32)
    sm.set_stream(stream.cuda_stream)
    sm.set_state(U0)
    _warm(dg, torch, sm, dt, 3)
    barrier()
    torch.cuda.synchronize()
    ms_mixed = max_over_ranks(_timed_steps(dg, torch, sm, stream, dt, args.steps))
    value_mixed = replica_rate(world, dof_stage, 4, args.steps, ms_mixed)
    stage_ms_mixed, trace_ms_mixed = _stage_kernel_ms(dg, sm, U0, dt, reps)
    # the same mixed form with its volume contractions on the tensor cores
    sm.set_step_form(dg.STEP_GAUSS_TC)
    sm.set_state(U0)
    _warm(dg, torch, sm, dt, 3)
    barrier()
    torch.cuda.synchronize()
    ms_tc = max_over_ranks(_timed_steps(dg, torch, sm, stream, dt, args.steps))
    stage_ms_tc, _ = _stage_kernel_ms(dg, sm, U0, dt, reps)
    sm.close()

    # ---- accuracy of the mixed form against the FP64 form after many steps
    acc = None
    if rank == 0 and args.accuracy_steps > 0:
        out = {}
        for prec in (dg.FP64, dg.MIXED_FP32):
            with dg.Solver(mesh, dg.Params.from_array(prm), prec) as sa:
                sa.set_state(U0)
                sa.step(dg.RK4, dt, args.accuracy_steps, norms=False)
                out[prec] = sa.get_state()
        err = float(np.linalg.norm(out[dg.MIXED_FP32] - out[dg.FP64]) / np.linalg.norm(out[dg.FP64]))
        acc = {"steps": args.accuracy_steps, "rel_l2_mixed_vs_fp64": err}

    # ---- adjoint: one reverse RK4 step against one forward step at this
    # workload, and the adjoint configuration's full gradient
    adj = None
    if rank == 0 and args.adjoint_steps > 0:
        with dg.Solver(mesh, dg.Params.from_array(prm), dg.FP64) as sa:
            sa.set_stream(stream.cuda_stream)
            rev_ms, rev_launches = _reverse_step_ms(dg, torch, sa, stream, U0, dt, reps)
            sweep_ms = _reverse_sweep_ms(dg, torch, sa, stream, U0, dt, 20)
            # the forward step the reverse step undoes: the recorded runs step
            # the nodal form
            sa.set_step_form(dg.STEP_NODAL)
            sa.set_state(U0)
            _warm(dg, torch, sa, dt, 3)
            nodal_ms = _timed_steps(dg, torch, sa, stream, dt, min(args.steps, 20)) / min(args.steps, 20)
        adj = {"reverse_step_ms": rev_ms, "forward_step_ms": ms / args.steps,
               "reverse_over_forward": rev_ms / (ms / args.steps),
               "sweep_reverse_step_ms": sweep_ms, "sweep_steps": 20,
               "sweep_reverse_over_forward": sweep_ms / (ms / args.steps), "forward_step_nodal_ms": nodal_ms,
               "reverse_over_nodal_forward": rev_ms / nodal_ms, "reverse_step_launches": rev_launches,
               "config": _adjoint_config(dg, torch, args.adjoint_steps, (args.adjoint_steps, 20, -1))}

    config3 = (_config3_block(dg, torch, min(args.steps, 20), args.config3_accuracy_steps)
               if rank == 0 and not args.no_config3 else None)
    curved = _curved_block(dg, torch, min(args.steps, 20)) if rank == 0 and not args.no_curved else None
    heat = _heat_block(dg, torch, min(args.steps, 20)) if rank == 0 and not args.no_heat else None
    channel = _channel_block(dg, torch, min(args.steps, 20)) if rank == 0 and not args.no_channel else None
    geometry = _geometry_block(dg, torch) if rank == 0 and not args.no_geometry else None
    ckpt = _checkpoint_block(dg) if rank == 0 and not args.no_checkpoint else None
    refcuda = _reference_cuda_block() if rank == 0 and not args.no_reference_cuda else None
    cpu_cfg = (_cpu_configs_block() if rank == 0 and not args.no_cpu_baseline and world == 1 else None)
    chadj = (_channel_adjoint_block(dg, torch, args.channel_adjoint_steps)
             if rank == 0 and not args.no_channel and args.channel_adjoint_steps > 0 else None)

    alg_bytes = (200 * nb + 80) * N_EL ** 3  # fused RK4 stage minimum, per element 200 nb + 80 B
    peak, peak_src = _hbm_peak()
    achieved = alg_bytes / (stage_ms * 1e-3) / 1e9
    achieved_mixed = alg_bytes / (stage_ms_mixed * 1e-3) / 1e9
    barrier()

    if rank == 0:
        cpu = None
        if not args.no_cpu_baseline and world == 1:
            import oracle
            if oracle.reference() is not None:
                procs, physical = host_cores()
                rate, _ = cpu_rate(1, REF_BLOCK, procs)
                cpu = {"value": rate, "unit": UNIT, "cores": procs, "physical_cores": physical, "kind": "reference",
                       "sample": f"{procs} concurrent reference processes, each 1 RK4 step on a {REF_BLOCK}^3 "
                                 f"block of the TGV mesh (same per-element work)"}
        prof = {}
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            prof = json.load(open(tpath))
        traffic = prof.get("stage_kernel_bytes_per_launch")
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "kernel": "wstage_kernel<4,double>", "kernel_ms": stage_ms,
                "trace_kernel_ms": trace_ms, "algorithmic_bytes_per_launch": alg_bytes, "peak_source": peak_src}
        fp64_flop = prof.get("stage_kernel_fp64_flop_per_launch")
        if fp64_flop:  # executed FP64 arithmetic (ncu instruction counts, scaled to the launch)
            rate = fp64_flop / (stage_ms * 1e-3) / 1e12
            roof["fp64_executed_tflops"] = rate
            roof["fp64_peak_tflops"] = FP64_PEAK_TFLOPS
            roof["fp64_frac"] = rate / FP64_PEAK_TFLOPS
            roof["fp64_peak_source"] = FP64_PEAK_SOURCE
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config(),
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "warmup_steps_run": warm_run,
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": U0.size * 8,
                    "d2h_bytes_per_step": U0.size * 8 + 8,
                    "call": "dgb_step_host_async per step, dgb_synchronize at the end (copies overlapped)",
                    "sync_call_value": e2e_sync,
                    "set_step_get_value": e2e_plain},
            "gpu_launches": int(launches),
            "roofline": roof,
            "mixed": {"value": value_mixed, "unit": UNIT, "ms_per_step": ms_mixed / args.steps,
                      "speedup_vs_fp64": value_mixed / value, "stage_kernel_ms": stage_ms_mixed,
                      "trace_kernel_ms": trace_ms_mixed,
                      "roofline": {"bound": "hbm", "achieved": achieved_mixed, "peak": peak, "unit": "GB/s",
                                   "frac": achieved_mixed / peak, "algorithmic_bytes_per_launch": alg_bytes},
                      "dtype": "f32 contractions/fluxes, f64 geometry/inverse mass/RK state",
                      "accuracy": acc,
                      "tensor_core": {"what": "volume contractions on tcgen05 (kind::tf32, 3 TF32 products, "
                                              "FP32 accumulation), one element per 128-thread CTA",
                                      "ms_per_step": ms_tc / args.steps,
                                      "value": replica_rate(world, dof_stage, 4, args.steps, ms_tc),
                                      "speedup_vs_fp64": (ms / ms_tc), "stage_kernel_ms": stage_ms_tc,
                                      "stage_vs_fp32x2_stage": stage_ms_tc / stage_ms_mixed}},
            "adjoint": adj,
            "config3": config3,
            "curved": curved,
            "heat": heat,
            "channel": channel,
            "geometry": geometry,
            "channel_adjoint": chadj,
            "checkpoint_cadence": ckpt,
            "reference_cuda": refcuda,
            "cpu_baseline_configs": cpu_cfg,
            "clocks": clocks,
        }
        if cpu:
            out["cpu_baseline"] = cpu
        # the headline figures again, short, at the end of the line
        head = {"fp64_value": value, "fp64_stage_frac": achieved / peak,
                "mixed_speedup_32_p3": value_mixed / value,
                "mixed_rel_l2_1000_32_p3": acc["rel_l2_mixed_vs_fp64"] if acc else None}
        if config3:
            head["mixed_speedup_48_p4"] = config3["speedup_mixed_vs_fp64"]
            head["mixed_rel_l2_48_p4"] = config3.get("accuracy", {}).get("rel_l2_mixed_vs_fp64")
        if adj:
            head["adjoint_reverse_over_forward"] = adj["reverse_over_forward"]
            head["adjoint_sweep_reverse_over_forward"] = adj["sweep_reverse_over_forward"]
            head["adjoint_config_backward_over_forward"] = {
                str(b["slots"]): round(b["backward_over_plain_forward"], 3) for b in adj["config"]["budgets"]}
            head["adjoint_config_fd_rel_l2"] = adj["config"]["fd_full"]["rel_l2"]
        if chadj:
            head["channel_grad_rel_err_fp64"] = chadj["rel_err_fp64_adjoint_vs_fd"]
            head["channel_grad_rel_err_mixed"] = chadj["rel_err_mixed_forward_vs_fd"]
        out["headline"] = head
        print(json.dumps(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-curved", action="store_true", help="skip the curved-mesh block")
    ap.add_argument("--no-heat", action="store_true", help="skip the heat-conduction block")
    ap.add_argument("--no-channel", action="store_true", help="skip the channel (isothermal walls) block")
    ap.add_argument("--no-geometry", action="store_true", help="skip the set-up (geometry build) timing")
    ap.add_argument("--channel-adjoint-steps", type=int, default=500,
                    help="TVD-RK3 steps of the channel adjoint block (0 or --no-channel skips it)")
    ap.add_argument("--nel", type=int, default=N_EL, help="elements per direction (profiling runs use fewer)")
    ap.add_argument("--p", type=int, default=P_ORD, help="solution order of the workload (profiling runs)")
    ap.add_argument("--reverse-steps-only", action="store_true",
                    help="only time reverse RK4 steps at the --nel workload (profiling the adjoint kernels)")
    ap.add_argument("--adjoint-steps", type=int, default=400,
                    help="RK4 steps of the adjoint configuration (0 skips the adjoint block)")
    ap.add_argument("--accuracy-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 accuracy check (0 skips it)")
    ap.add_argument("--no-config3", action="store_true", help="skip the 48^3 p = 4 block")
    ap.add_argument("--no-checkpoint", action="store_true", help="skip the driver's checkpoint-cadence timing")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="skip timing the reference's own GPU driver beside dgb")
    ap.add_argument("--config3-accuracy-steps", type=int, default=1000,
                    help="steps of the 48^3 p = 4 mixed-vs-FP64 accuracy and kinetic-energy check (0 skips it)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    globals()["N_EL"] = args.nel
    globals()["P_ORD"] = args.p
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.reverse_steps_only:
        run_reverse_steps(args)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    run_ours(args, rank, world, local_rank)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
