"""Benchmark: DOF-updates/s of the nodal-DG SSPRK(5,2) stepper on B200.

Workload (one "step" = one SSPRK(5,2) time step, 5 right-hand sides, over the
whole mesh): 2D compressible Euler isentropic vortex (gamma 1.4, strength 5,
centre (5,5)) on the periodic [0,10]^2, 256 x 256 jittered vertex grid
(K = 130,050 triangles), order N = 4 (Np = 15), Lax-Friedrichs (Rusanov) flux,
CFL 0.5, 4 conserved fields.  DOF = K * Np * 4; one DOF-update = one DOF
advanced by one full step.  Synthetic seeded mesh and closed-form initial state.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed|auto]
    python bench.py --impl reference ...   # the CPU reference arm

Multi-GPU (torchrun): one periodic mesh of N x the single-GPU workload split
into one strip per rank; per stage the ranks exchange the traces of their cut
faces (NCCL point-to-point) and per step MAX-reduce the wave speed (weak
scaling; ``--replicas`` runs independent instances instead); the time is the
max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DOF-updates/s"
WORKLOAD = "euler_vortex_N4_K130050"


def workload_name(N: int, K: int) -> str:
    return f"euler_vortex_N{N}_K{K}"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="auto", choices=["auto", "fp64", "mixed"])
    ap.add_argument("--n", type=int, default=256, help="vertex grid size (256: K = 130,050)")
    ap.add_argument("--order", type=int, default=4, help="polynomial order N of the vortex workload (2..5)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-l2-500", action="store_true", help="skip the 500-step mixed vs float64 comparison")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the discrete-adjoint measurement")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble measurement")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the advection (K = 1,922) and Maxwell TM (N = 5) configurations")
    ap.add_argument("--maxwell-n", type=int, default=512, help="vertex grid of the Maxwell TM configuration")
    ap.add_argument("--maxwell-steps", type=int, default=1000)
    ap.add_argument("--replicas", action="store_true",
                    help="N>1: independent replicas instead of one partitioned mesh")
    ap.add_argument("--partitioned", action="store_true",
                    help="run the partitioned (multi-GPU) arm even at N=1 (one part, no peers)")
    ap.add_argument("--ensemble-steps", type=int, default=20)
    ap.add_argument("--adjoint-dirs", type=int, default=32,
                    help="random directions of the adjoint's finite-difference check")
    ap.add_argument("--rhs-only", type=int, default=0,
                    help="profiling driver: set up the workload, run this many RHS evaluations, exit")
    ap.add_argument("--steps-only", type=int, default=0,
                    help="profiling driver: set up the workload, advance this many SSPRK steps, exit")
    ap.add_argument("--vjp-only", type=int, default=0,
                    help="profiling driver: set up the workload, evaluate this many adjoint right-hand sides, exit")
    ap.add_argument("--fp64-kernels", type=int, default=0, choices=[0, 1, 2],
                    help="profiling drivers: the float64 stage form (0 three kernels, 1 fused, 2 by mesh size)")
    return ap.parse_args()


def rhs_only(args):
    """Set up the benchmark workload and evaluate the RHS a few times (for ncu)."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    p = problems.euler_vortex(n=args.n, N=args.order, fields=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=0)
    s.set_fp64_kernels(args.fp64_kernels)
    x, y = s.node_coords()
    u = torch.from_numpy(np.ascontiguousarray(p.ic(x, y))).cuda()
    out = torch.empty_like(u)
    prec = "fp64" if args.precision == "auto" else args.precision
    for _ in range(args.rhs_only):
        s.step(0.0, 0.0, u, out, precision=prec)
    torch.cuda.synchronize()
    print(json.dumps({"rhs_only": args.rhs_only, "K": s.K, "precision": prec,
                      "checksum": float(out.abs().sum().item())}))
    s.close()
    return 0


def vjp_only(args):
    """Set up the benchmark workload and evaluate the adjoint of its right-hand
    side a few times (for ncu: the discrete adjoint's stage kernels)."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    p = problems.euler_vortex(n=args.n, N=args.order, fields=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=0)
    x, y = s.node_coords()
    u = torch.from_numpy(np.ascontiguousarray(p.ic(x, y))).cuda()
    w = torch.from_numpy(np.random.default_rng(0).standard_normal(u.shape)).cuda()
    out = torch.empty_like(u)
    for _ in range(args.vjp_only):
        s.rhs_vjp(0.0, u, w, out)
    torch.cuda.synchronize()
    print(json.dumps({"vjp_only": args.vjp_only, "K": s.K, "checksum": float(out.abs().sum().item())}))
    s.close()
    return 0


def steps_only(args):
    """Set up the benchmark workload and advance it a few steps (for ncu: the
    stepper's stage-mode launches)."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    p = problems.euler_vortex(n=args.n, N=args.order, fields=4)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=0)
    s.set_fp64_kernels(args.fp64_kernels)
    x, y = s.node_coords()
    s.set_state(np.ascontiguousarray(p.ic(x, y)))
    prec = "fp64" if args.precision == "auto" else args.precision
    t, dt = s.advance(args.steps_only, 0.0, s.init_dt(), precision=prec)
    torch.cuda.synchronize()
    print(json.dumps({"steps_only": args.steps_only, "K": s.K, "precision": prec, "t": t,
                      "checksum": float(np.abs(s.get_state()).sum())}))
    s.close()
    return 0


def adjoint_measure(args, device: int):
    """The discrete-adjoint configuration: Euler vortex on a 128 x 128 vertex
    grid (K = 32,258), N = 3, 400 fixed SSPRK(5,2) steps, checkpoints every 20.
    J = 0.5 ||U(T) - U_target||^2 with U_target the float64 forward of the
    vortex and U(0) = vortex + N(0, 1e-3^2) (seeded).  Reports the time of the
    forward (with checkpoints) and of the backward (segment re-runs + reverse
    stages), the derivative memory, and the gradient checked against central
    finite differences and the forward-mode derivative on random directions."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    p = problems.euler_vortex(n=128, N=3)
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=device)
    x, y = s.node_coords()
    u_ic = np.ascontiguousarray(p.ic(x, y))
    s.set_state(u_ic)
    dt = s.init_dt()
    nsteps, every = 400, 20
    s.forward_fixed(nsteps, 0.0, dt, every)
    target = torch.from_numpy(s.get_state()).cuda(device)
    rng = np.random.default_rng(0)
    u0 = torch.from_numpy(u_ic + 1e-3 * rng.standard_normal(u_ic.shape)).cuda(device)
    uT = torch.empty_like(u0)
    grad = torch.empty_like(u0)

    def J(u):
        s.set_state(u)
        s.forward_fixed(nsteps, 0.0, dt, every)
        s.get_state(uT)
        return 0.5 * float(((uT - target) ** 2).sum())

    J(u0)
    s.backward(uT - target, out=grad)  # warm-up: buffers allocated
    torch.cuda.synchronize()
    fwd, bwd = [], []
    for _ in range(3):
        s.set_state(u0)
        t0 = time.perf_counter()
        s.forward_fixed(nsteps, 0.0, dt, every)
        t1 = time.perf_counter()
        s.get_state(uT)
        gT = uT - target
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        s.backward(gT, out=grad)
        t3 = time.perf_counter()
        fwd.append(t1 - t0)
        bwd.append(t3 - t2)
    g = grad.cpu().numpy()
    gT_host = (uT - target).cpu().numpy()
    fd_err, tan_err = [], []
    drng = np.random.default_rng(1)
    for i in range(args.adjoint_dirs):
        d = torch.from_numpy(drng.standard_normal(u_ic.shape)).cuda(device)
        eps = 1e-6
        fd = (J(u0 + eps * d) - J(u0 - eps * d)) / (2 * eps)
        ga = float(np.vdot(g, d.cpu().numpy()))
        fd_err.append(abs(ga - fd) / abs(fd))
        if i < 4:
            s.set_state(u0)
            du = s.tangent(nsteps, 0.0, dt, d)
            gt = float(np.vdot(gT_host, du.cpu().numpy()))
            tan_err.append(abs(ga - gt) / abs(gt))
    two_level_memory = s.adjoint_memory()
    revolve = {}
    for snaps in (20, 5):
        s.set_state(u0)
        s.forward_revolve(nsteps, 0.0, dt, snaps)
        s.get_state(uT)
        s.backward(uT - target, out=grad)  # warm-up: slots sized
        torch.cuda.synchronize()
        rf, rb = [], []
        for _ in range(3):
            s.set_state(u0)
            t0 = time.perf_counter()
            s.forward_revolve(nsteps, 0.0, dt, snaps)
            t1 = time.perf_counter()
            s.get_state(uT)
            gT = uT - target
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            s.backward(gT, out=grad)
            t3 = time.perf_counter()
            rf.append(t1 - t0)
            rb.append(t3 - t2)
        gr = grad.cpu().numpy()
        revolve[str(snaps)] = {
            "snapshots": snaps, "forward_ms": 1000 * float(np.median(rf)), "backward_ms": 1000 * float(np.median(rb)),
            "adjoint_over_forward": float(np.median(rb) / np.median(rf)),
            "recomputed_steps": s.recomputed_steps(),
            "derivative_memory_mb": s.adjoint_memory() / 2**20,
            "grad_equals_two_level": bool(np.array_equal(gr, g)),
            "grad_max_abs_diff_vs_two_level": float(np.abs(gr - g).max()),
        }
    nU = s.K * s.Np * s.m * 8
    out = {
        "config": {"workload": "euler_vortex_N3_K32258_400steps", "K": s.K, "N": 3, "fields": s.m, "steps": nsteps,
                   "checkpoint_every": every, "dt": dt, "functional": "0.5 ||U(T) - U_target||^2"},
        "forward_ms": 1000 * float(np.median(fwd)), "backward_ms": 1000 * float(np.median(bwd)),
        "adjoint_over_forward": float(np.median(bwd) / np.median(fwd)),
        "derivative_memory_mb": two_level_memory / 2**20,
        "state_mb": nU / 2**20,
        "fd_directions": args.adjoint_dirs, "fd_max_rel_err": max(fd_err) if fd_err else None,
        "tangent_max_rel_err": max(tan_err) if tan_err else None,
        "revolve": revolve,
        "how": "wall clock around the synchronous C-ABI calls (median of 3); float64; fixed dt; revolve budgets "
               "count the initial state's slot",
    }
    s.close()
    return out


def _device_run(s, stream, U0, dt0, prec: str, steps: int, warmup: int = 3):
    """ms for `steps` steps of the resident state from U0 at t = 0 (CUDA events on
    the handle's stream, after `warmup` untimed steps from U0), and (t, dt)."""
    import torch
    s.set_state(U0)
    s.advance(warmup, 0.0, dt0, precision=prec)
    s.set_state(U0)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        s.advance_async(steps, 0.0, dt0, precision=prec)
        e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), s.time()


def _cpu_rate(o, U, steps: int, threads: int):
    """DOF-updates/s of the oracle on `threads` threads over `steps` steps of U
    (advanced in place), and the seconds taken."""
    o.set_threads(threads)
    dt = o.init_dt(U)
    t0 = time.perf_counter()
    n, _, _ = o.run(U, steps, 0.0, dt)
    return n, time.perf_counter() - t0


def advection_measure(args, device: int, cpu: bool):
    """Scalar advection by (1, 0.5) of the Gaussian exp(-r^2/0.01) on the periodic
    unit square, jittered 32 x 32 vertex grid (K = 1,922), N = 3, CFL 0.5, 200
    steps of the adaptive SSPRK(5,2) stepper: both GPU forms, the mixed form's
    error against float64, and the CPU oracle on the same run (all host threads,
    200 steps: its rate and the float64 GPU state's relative L2 against it) and
    on one thread (a 10-step sample)."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    p = problems.advection(n=32, N=3)
    stream = torch.cuda.Stream()
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=device, stream=stream.cuda_stream)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    steps = 200
    dofs = s.K * s.Np * s.m
    out = {"config": {"workload": "advection_N3_K1922_200steps", "K": s.K, "N": p.N, "fields": 1,
                      "velocity": [1.0, 0.5], "flux": "LF", "cfl": p.cfl, "steps": steps}}
    ends = {}
    for prec in ("fp64", "mixed"):
        ms, (t, dt) = _device_run(s, stream, U0, dt0, prec, steps)
        ends[prec] = s.get_state()
        out[prec] = {"value": dofs * steps / (ms / 1000.0), "ms_per_step": ms / steps, "t_end": t}
    out["l2_mixed_vs_fp64"] = float(np.linalg.norm(ends["mixed"] - ends["fp64"]) / np.linalg.norm(ends["fp64"]))
    # the mesh is one wave of tiles: the fused float64 stage (one launch per
    # stage instead of three) is the faster form here
    s.set_fp64_kernels(1)
    ms, (t, dt) = _device_run(s, stream, U0, dt0, "fp64", steps)
    out["fp64_fused_stage"] = {"value": dofs * steps / (ms / 1000.0), "ms_per_step": ms / steps, "t_end": t,
                               "l2_vs_fp64": float(np.linalg.norm(s.get_state() - ends["fp64"]) /
                                                   np.linalg.norm(ends["fp64"]))}
    s.set_fp64_kernels(0)
    # the configuration names an upwind flux; Apollo's advection flux is
    # Lax-Friedrichs with max(|ux|, |uy|) (the parity runs above), and the
    # upwind flux (dissipation |n.u|) is this library's extension
    su = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=device, stream=stream.cuda_stream,
                   numerical_flux="upwind")
    su.set_state(U0)
    ms, (t, dt) = _device_run(su, stream, U0, dt0, "fp64", steps)
    Uup = su.get_state()
    out["fp64_upwind"] = {"value": dofs * steps / (ms / 1000.0), "ms_per_step": ms / steps, "t_end": t}
    su.close()
    if cpu:
        from oracle import oracle as orc
        threads = os.cpu_count() or 1
        o = orc.Oracle(p.mesh, p.N, orc.EQ_ADVECTION, p.eq_params, cfl=p.cfl)
        Uc = U0.copy()
        n, el = _cpu_rate(o, Uc, steps, threads)
        out["cpu_all_cores"] = {"value": dofs * n / el, "cores": threads, "steps": n, "seconds": el}
        out["l2_fp64_gpu_vs_cpu_oracle"] = float(np.linalg.norm(ends["fp64"] - Uc) / np.linalg.norm(Uc))
        ou = orc.Oracle(p.mesh, p.N, orc.EQ_ADVECTION, tuple(p.eq_params)[:3] + (orc.NF_UPWIND,), cfl=p.cfl)
        ou.set_threads(threads)
        Uu = U0.copy()
        ou.run(Uu, steps, 0.0, dt0)
        out["fp64_upwind"]["l2_vs_cpu_oracle"] = float(np.linalg.norm(Uup - Uu) / np.linalg.norm(Uu))
        n1, el1 = _cpu_rate(o, U0.copy(), 10, 1)
        out["cpu_1_thread"] = {"value": dofs * n1 / el1, "cores": 1, "steps": n1, "seconds": el1}
    s.close()
    return out


def maxwell_measure(args, device: int, cpu: bool):
    """Maxwell TM cavity (Ez, Bx, By; c = 1) on the unit square with Apollo's
    mirror wall condition (maxwellTransverseMagneticBC), jittered 512 x 512
    vertex grid (K = 522,242), N = 5, CFL 0.5, 1000 steps from the mode
    Ez = sin(pi x) sin(pi y): both GPU forms (their device time over the 1000
    steps), the drift of the energy 1/2 int (Ez^2 + Bx^2 + By^2) dA, the
    relative L2 error against the exact mode at the time reached, the mixed form
    against float64; the CPU oracle's rate on bounded samples (one step of the
    same physics on a 128 x 128 grid on all host threads, one step on a 48 x 48
    grid on one thread)."""
    import torch
    from apollo_b200 import NodalDG2d, problems
    n = args.maxwell_n
    p = problems.maxwell_tm(n=n, N=5)
    stream = torch.cuda.Stream()
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, device=device,
                  stream=stream.cuda_stream)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()
    steps = args.maxwell_steps
    dofs = s.K * s.Np * s.m
    e0 = 0.5 * float(np.sum(s.square_integrals(U0)))
    out = {"config": {"workload": f"maxwell_tm_N5_K{s.K}_{steps}steps", "K": s.K, "N": p.N, "fields": 3,
                      "bc": "maxwellTransverseMagneticBC (PEC)", "flux": "LF", "cfl": p.cfl, "steps": steps},
           "energy_0": e0}
    ends = {}
    for prec in ("fp64", "mixed"):
        ms, (t, dt) = _device_run(s, stream, U0, dt0, prec, steps, warmup=2)
        U = s.get_state()
        ends[prec] = U
        ex = p.exact(x, y, t)
        e1 = 0.5 * float(np.sum(s.square_integrals(U)))
        out[prec] = {"value": dofs * steps / (ms / 1000.0), "ms_per_step": ms / steps, "t_end": t,
                     "energy_drift_rel": (e1 - e0) / e0,
                     "l2_vs_exact_mode": float(np.linalg.norm(U - ex) / np.linalg.norm(ex))}
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    out["l2_mixed_vs_fp64"] = float(np.linalg.norm(ends["mixed"] - ends["fp64"]) / np.linalg.norm(ends["fp64"]))
    # the configuration names an upwind flux; Apollo's Maxwell flux is
    # Lax-Friedrichs (the runs above), the exact upwind flux (no dissipation
    # on the normal magnetic field) is this library's extension
    su = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, bcs=p.bcs, device=device,
                   stream=stream.cuda_stream, numerical_flux="upwind")
    su.set_state(U0)
    ms, (t, dt) = _device_run(su, stream, U0, dt0, "fp64", steps, warmup=2)
    U = su.get_state()
    ex = p.exact(x, y, t)
    e1 = 0.5 * float(np.sum(su.square_integrals(U)))
    out["fp64_upwind"] = {"value": dofs * steps / (ms / 1000.0), "ms_per_step": ms / steps, "t_end": t,
                          "energy_drift_rel": (e1 - e0) / e0,
                          "l2_vs_exact_mode": float(np.linalg.norm(U - ex) / np.linalg.norm(ex))}
    su.close()
    if cpu:
        from oracle import oracle as orc
        threads = os.cpu_count() or 1
        for key, ng, th in (("cpu_all_cores", 128, threads), ("cpu_1_thread", 48, 1)):
            q = problems.maxwell_tm(n=ng, N=5)
            o = orc.Oracle(q.mesh, q.N, orc.EQ_MAXWELL, (1.0, 0.0, 0.0), bcs=((orc.BC_TM, ()),), cfl=q.cfl)
            xo, yo = o.node_coords()
            U8 = np.zeros((q.mesh.K, o.Np, 8))
            U8[..., 2:5] = q.ic(xo, yo)
            nst, el = _cpu_rate(o, U8, 1, th)
            out[key] = {"value": q.mesh.K * o.Np * 3 * nst / el, "cores": th, "steps": nst, "seconds": el,
                        "sample": f"{nst} step on a {ng}x{ng} vertex grid (K={q.mesh.K}), N = 5, 8 Apollo fields"}
    s.close()
    return out


def apollo_cpu_extra(procs: int | None = None):
    """Apollo's own code (where it is built) on the other configurations'
    problems, bounded samples: the TM cavity at N = 5 and a walled Gaussian
    advection at N = 3 on every host core, one process per core, and the
    vortex at N = 4 on one core.  DOF counts the physical fields (3, 1, 4)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    if not orc.RefDriver.available():
        return None
    import multiprocessing as mp
    procs = procs or _host_cores()
    res = {}
    for key, case, n, m, steps, pp in (("maxwell_tm_N5", "tm", 24, 3, 2, procs),
                                       ("advection_N3", "advection", 32, 1, 4, procs),
                                       ("euler_vortex_N4_1_core", "vortex", APOLLO_SAMPLE_N, 4, 2, 1)):
        with mp.get_context("spawn").Pool(pp) as pool:
            out = pool.map(_apollo_steps, [(n, steps, 1, case)] * pp)
        el = max(o[0] for o in out)
        K, Np = out[0][1], out[0][2]
        res[key] = {"value": pp * K * Np * m * steps / el, "cores": pp, "K_per_process": K, "steps": steps,
                    "seconds": el, "kind": "reference",
                    "sample": f"{steps} SSPRK(5,2) steps per process through Apollo's own right-hand-side code "
                              f"on a {n}x{n} vertex grid (K={K}), {pp} process(es)"}
    return res


def cpu_extra(threads: int):
    """CPU oracle rates the single-GPU line reports beside its own numbers: the
    Euler vortex at N = 4 on one thread (one step of a 64 x 64 grid), and the
    float64 forward of the adjoint configuration (Euler vortex, N = 3, 128 x 128
    grid, K = 32,258) on all host threads (two steps), with the 400-step forward
    time that rate implies."""
    from apollo_b200 import problems
    from oracle import oracle as orc
    res = {}
    p = problems.euler_vortex(n=64, N=4, fields=5)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_EULER, p.eq_params, cfl=p.cfl)
    x, y = o.node_coords()
    n, el = _cpu_rate(o, np.ascontiguousarray(p.ic(x, y)), 1, 1)
    res["euler_vortex_N4_cpu_1_thread"] = {"value": p.mesh.K * o.Np * 4 * n / el, "cores": 1, "steps": n,
                                           "seconds": el, "sample": f"{n} step, 64x64 vertex grid (K={p.mesh.K})"}
    p = problems.euler_vortex(n=128, N=3, fields=5)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_EULER, p.eq_params, cfl=p.cfl)
    x, y = o.node_coords()
    n, el = _cpu_rate(o, np.ascontiguousarray(p.ic(x, y)), 2, threads)
    res["adjoint_config_cpu_forward"] = {"ms_per_step": 1000 * el / n, "forward_400_steps_s": 400 * el / n,
                                         "cores": threads, "steps": n,
                                         "sample": f"{n} steps, 128x128 vertex grid (K={p.mesh.K}), N = 3"}
    return res


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


# --------------------------------------------------------------- CPU arm ----
APOLLO_SAMPLE_N = 48  # vertex grid of each process's sample (K = 4,418 at N = 4)


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _apollo_steps(job):
    """One process of the reference arm: Apollo's own right-hand-side code
    (compiled unmodified into oracle/_ref) stepping one of its example
    problems on an n x n vertex grid: the isentropicVortex example on
    [0, 10]^2 at order 4 (case "vortex"), the transverseMagnetic cavity on
    [0, 1]^2 at order 5 ("tm"), or a Gaussian advected on [0, 1]^2 at order 3
    ("advection"); returns the seconds of the timed steps, the elements and
    the nodes per element."""
    n, steps, warmup = job[:3]
    case = job[3] if len(job) > 3 else "vortex"
    sys.path.insert(0, ROOT)
    from apollo_b200.mesh import jittered_square
    from oracle import oracle as orc
    if case == "vortex":
        mesh = jittered_square(n, (0.0, 0.0), (10.0, 10.0), seed=0, periodic=False, wall_tag=1)
        r = orc.apollo_vortex_driver(mesh, 4, 0.5)
    else:
        mesh = jittered_square(n, seed=0, periodic=False, wall_tag=1)
        r = (orc.apollo_tm_driver if case == "tm" else orc.apollo_advection_driver)(mesh, 5 if case == "tm" else 3,
                                                                                     0.5)
    u, dt = r.init(0.0)
    u, t, dt = r.run(u, warmup, 0.0, dt)
    t0 = time.perf_counter()
    r.run(u, steps, t, dt)
    return time.perf_counter() - t0, mesh.K, r.Np


def apollo_cpu_rate(steps: int, warmup: int, procs: int | None = None):
    """DOF-updates/s of Apollo's own code on the host: one process per core
    (as Apollo runs one MPI rank per core), each stepping its own sample
    with no exchange between them (which only favours the reference), timed
    together.  None where Apollo's code is not built (oracle/_ref)."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    if not orc.RefDriver.available():
        return None
    import multiprocessing as mp
    procs = procs or _host_cores()
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_apollo_steps, [(APOLLO_SAMPLE_N, steps, warmup)] * procs)
    el = max(r[0] for r in res)
    K, Np = res[0][1], res[0][2]
    return {"value": procs * K * Np * 4 * steps / el, "seconds": el, "cores": procs, "K": K,
            "sample": f"{steps} SSPRK(5,2) steps per process through Apollo's own right-hand-side code "
                      f"(WxNodalDG2dMethod with its geometry and cubature, compiled unmodified; the stage "
                      f"arithmetic as PETSc's TSSSP documents it), its isentropicVortex example on a "
                      f"{APOLLO_SAMPLE_N}x{APOLLO_SAMPLE_N} vertex grid (K={K}, N = 4, walls carrying the exact "
                      f"vortex), {procs} processes, one per host core"}


def cpu_sample(n_sample: int = 256, steps: int = 8, threads: int | None = None):
    """Time the CPU oracle (all host threads) on a bounded sample of the workload: the
    benchmark mesh itself (256 x 256 vertex grid, K = 130,050) for a few steps (about
    10 s of CPU work on 16 threads)."""
    from apollo_b200 import problems
    from oracle import oracle as orc
    threads = threads or os.cpu_count() or 1
    p = problems.euler_vortex(n=n_sample, fields=5)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_EULER, p.eq_params, cfl=p.cfl)
    o.set_threads(threads)
    x, y = o.node_coords()
    U = np.ascontiguousarray(p.ic(x, y))
    dt = o.init_dt(U)
    o.rhs(U)  # warm caches
    t0 = time.perf_counter()
    n, t, dt = o.run(U, steps, 0.0, dt)
    el = time.perf_counter() - t0
    dofs = p.mesh.K * o.Np * 4
    return {
        "value": dofs * n / el, "unit": METRIC, "cores": threads, "kind": "port",
        "sample": f"{n} SSPRK(5,2) steps of the same vortex problem on a {n_sample}x{n_sample} vertex grid "
                  f"(K={p.mesh.K}), CPU oracle (C++ restatement of Apollo's RHS loop, float64, 5 Euler fields "
                  f"as Apollo carries them), {threads} threads",
        "seconds": el,
    }


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    orc.build(with_ref=False)
    ref = apollo_cpu_rate(args.steps, args.warmup)
    if ref is not None:
        value = ref["value"]
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * ref["seconds"] / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "sample_K_per_process": ref["K"], "N": 4, "fields": 4, "flux": "LF"},
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": ref["cores"], "kind": "reference",
                             "sample": ref["sample"]},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return 0
    # Apollo's code is not built here: the oracle's restatement of it
    from apollo_b200 import problems
    threads = os.cpu_count() or 1
    p = problems.euler_vortex(n=128, fields=5)
    o = orc.Oracle(p.mesh, p.N, orc.EQ_EULER, p.eq_params, cfl=p.cfl)
    o.set_threads(threads)
    x, y = o.node_coords()
    U = np.ascontiguousarray(p.ic(x, y))
    t, dt = 0.0, o.init_dt(U)
    for _ in range(args.warmup):
        _, t, dt = o.run(U, 1, t, dt)
    t0 = time.perf_counter()
    _, t, dt = o.run(U, args.steps, t, dt)
    el = time.perf_counter() - t0
    dofs = p.mesh.K * o.Np * 4
    value = dofs * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * el / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_K": p.mesh.K, "N": 4, "fields": 4, "flux": "LF"},
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"each step: one SSPRK(5,2) step of the vortex on a 128x128 vertex grid "
                                   f"(K={p.mesh.K}); Apollo's RHS algorithm restated in C++ (oracle), "
                                   f"{threads} threads"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# --------------------------------------------------------------- GPU arm ----
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join("/tmp", f"apollo_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.f.close()
        except Exception:
            pass

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and "Active" in r[5 + i] and "Not" not in r[5 + i]:
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def fp64_gemm_peak(device: int) -> float:
    """Float64 dense GEMM throughput of this GPU (TFLOP/s): cuBLAS DGEMM through
    torch.matmul on 4096^3 operands, best of 5 (CUDA events), the denominator of
    the float64 path's roofline (the measured peaks file has no float64 entry)."""
    import torch
    n = 4096
    a = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{device}")
    b = torch.randn(n, n, dtype=torch.float64, device=f"cuda:{device}")
    c = torch.empty_like(a)
    for _ in range(2):
        torch.matmul(a, b, out=c)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1000.0)
    del a, b, c
    return 2.0 * n ** 3 / best / 1e12


def profile_traffic():
    """DRAM bytes per launch of the dominant kernels from the committed ncu summary."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
    except Exception:
        return {}


def ensemble_measure(args, device: int):
    """The batched-ensemble configuration: 64 independent Euler vortices with
    seed-drawn element counts K uniform in [1000, 64000], orders N in {2..5}
    and strengths beta uniform in [1, 5] (seed 0).  The batch (one handle per
    order, one persistent launch per stage per order, one CUDA graph per step,
    grid shares picked by the autotuner) against the same instances advanced
    one by one through their own handles; aggregate DOF-updates/s, and per
    instance the error against the exact vortex and mixed against float64."""
    from collections import Counter
    from apollo_b200 import NodalDG2d, NodalDG2dBatch, problems
    ps = problems.euler_ensemble(count=64, k_range=(1000, 64000), seed=0)
    steps = args.ensemble_steps
    b = NodalDG2dBatch(ps[0].cfl, ps[0].equation, ps[0].eq_params, device=device)
    for p in ps:
        b.add_mesh(p.N, p.mesh)
    b.finalize()
    xy = [b.node_coords(i) for i in range(len(ps))]
    U0 = [np.ascontiguousarray(p.ic(x, y)) for p, (x, y) in zip(ps, xy)]
    dofs = sum(int(np.prod(b.shape(i))) for i in range(len(ps)))

    def reset():
        for i, u in enumerate(U0):
            b.set_state(i, u)

    reset()
    dt0 = b.init_dt()
    tune = b.autotune("mixed")
    res, ends = {}, {}
    for prec in ("mixed", "fp64"):
        reset()
        b.step(3, np.zeros(len(ps)), dt0, precision=prec)  # warm-up: graphs built
        reset()
        t0 = time.perf_counter()
        t_end, _ = b.step(steps, np.zeros(len(ps)), dt0, precision=prec)
        el = time.perf_counter() - t0
        res[prec] = {"value": dofs * steps / el, "ms_per_step": 1000 * el / steps}
        ends[prec] = ([b.get_state(i) for i in range(len(ps))], t_end)
    # one by one: each instance its own handle, advanced in turn
    singles = []
    for p, u in zip(ps, U0):
        h = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=device)
        h.set_state(u)
        singles.append(h)
    for prec in ("mixed", "fp64"):
        for h, u, d in zip(singles, U0, dt0):
            h.set_state(u)
            h.advance(3, 0.0, d, precision=prec)
            h.set_state(u)
        t0 = time.perf_counter()
        for h, d in zip(singles, dt0):
            h.advance(steps, 0.0, d, precision=prec)
        el = time.perf_counter() - t0
        res[prec]["one_by_one"] = {"value": dofs * steps / el, "ms_per_step": 1000 * el / steps}
        res[prec]["speedup_vs_one_by_one"] = res[prec]["value"] / res[prec]["one_by_one"]["value"]
    for h in singles:
        h.close()
    b.close()
    e_exact, e_mixed = [], []
    (Um, _), (U64, t64) = ends["mixed"], ends["fp64"]
    for i, (p, (x, y)) in enumerate(zip(ps, xy)):
        ex = p.exact(x, y, t64[i])
        e_exact.append(float(np.linalg.norm(Um[i] - ex) / np.linalg.norm(ex)))
        e_mixed.append(float(np.linalg.norm(Um[i] - U64[i]) / np.linalg.norm(U64[i])))
    return {
        "config": {"workload": "euler_vortex_ensemble_64", "instances": len(ps), "K_total": sum(p.mesh.K for p in ps),
                   "K_min": min(p.mesh.K for p in ps), "K_max": max(p.mesh.K for p in ps),
                   "orders": dict(sorted(Counter(p.N for p in ps).items())),
                   "beta_range": [min(p.meta["beta"] for p in ps), max(p.meta["beta"] for p in ps)],
                   "dofs": dofs, "steps": steps, "seed": 0},
        "unit": METRIC, "mixed": res["mixed"], "fp64": res["fp64"], "autotune_share_and_shape": {str(k): list(v) for k, v in tune.items()},
        "per_instance": {"l2_mixed_vs_exact": e_exact, "l2_mixed_vs_fp64": e_mixed,
                         "max_l2_mixed_vs_fp64": max(e_mixed), "max_l2_mixed_vs_exact": max(e_exact)},
        "how": "wall clock around the synchronous C-ABI calls (apollo_dg_batch_step; apollo_dg_step per "
               "instance for one by one), states resident, adaptive per-instance dt",
    }


def partitioned_arm(args, rank: int, world: int, local: int):
    """N > 1: one periodic mesh of world x (the single-GPU workload), [0,10] x
    [0,10 world] with an n x ((n-1) world + 1) vertex grid, split into one strip
    per rank by recursive coordinate bisection; per stage each rank exchanges
    the traces of its cut faces with its neighbours (NCCL point-to-point) and
    per step the wave speed is MAX-reduced (NCCL all-reduce).  Weak scaling:
    K = 130,050 elements per rank at n = 256."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from apollo_b200 import NodalDG2d, problems
    from apollo_b200.distributed import DistNodalDG2d, TorchComm, partition
    from apollo_b200.mesh import jittered_square
    dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    comm = TorchComm()
    n = args.n
    p = problems.euler_vortex(n=n, fields=4)
    mesh = jittered_square(n, (0.0, 0.0), (10.0, 10.0 * world), jitter=0.2, seed=0, periodic=True,
                           ny=(n - 1) * world + 1)
    part = partition(mesh, world)
    d = DistNodalDG2d(p.N, p.cfl, p.equation, p.eq_params, mesh, part, comm, device=local)
    x, y = d.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    d.set_state(U0)
    dt0 = d.init_dt()
    prec = "mixed" if args.precision in ("auto", "mixed") and "mixed" in d.block_bytes else "fp64"
    K_local = d.shape[0]
    dofs_all = mesh.K * d.shape[1] * d.shape[2]

    def timed(precision, steps, warmup):
        d.set_state(U0)
        t_w, dt_w = d.advance(warmup, 0.0, dt0, precision=precision)
        dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(d.torch_stream)
        d.advance(steps, t_w, dt_w, precision=precision)
        e1.record(d.torch_stream)
        e1.synchronize()
        torch.cuda.synchronize()
        tt = torch.tensor([e0.elapsed_time(e1)], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    with ClockSampler(local) as clk:
        ms = timed(prec, args.steps, args.warmup)
    clocks = clk.summary()
    value = dofs_all * args.steps / (ms / 1000.0)
    extra = {}
    if prec == "mixed":
        ms64 = timed("fp64", args.steps, args.warmup)
        extra["fp64"] = {"value": dofs_all * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps}

    e2e = None
    if not args.no_e2e:
        # per step: the rank's state from pinned host memory, one step, back to pinned host memory
        hU = torch.empty(d.shape, dtype=torch.float64, pin_memory=True)
        hU.numpy()[...] = U0
        hO = torch.empty(d.shape, dtype=torch.float64, pin_memory=True)
        t, dt = 0.0, dt0
        ne = max(3, min(args.steps, 50))
        for _ in range(2):
            d.set_state(hU.numpy())
            t, dt = d.advance(1, t, dt, precision=prec)
            d.get_state(hO.numpy())
        dist.barrier()
        t0 = time.perf_counter()
        for _ in range(ne):
            d.set_state(hU.numpy())
            t, dt = d.advance(1, t, dt, precision=prec)
            d.get_state(hO.numpy())
        el = time.perf_counter() - t0
        tt = torch.tensor([el], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        el = float(tt.item())
        nb = K_local * d.shape[1] * d.shape[2] * 8
        e2e = {"value": dofs_all * ne / el, "unit": METRIC, "h2d_bytes_per_step": nb * world,
               "d2h_bytes_per_step": nb * world, "steps": ne,
               "how": "wall clock, max over ranks; per step and rank: set_state (pinned H2D), one partitioned "
                      "step (5 trace exchanges + wave-speed all-reduce), get_state (pinned D2H)"}

    # the dominant kernel's roofline, from a whole-mesh handle of one rank's size
    roofline = None
    if rank == 0:
        s1 = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=local)
        xs, ys = s1.node_coords()
        s1.set_state(np.ascontiguousarray(p.ic(xs, ys)))
        kt = s1.kernel_times(10, precision=prec)
        peaks, peak_src = measured_peaks()
        K1, Np, M, Nf = s1.K, s1.Np, s1.m, 3 * s1.Ng
        if prec == "mixed":
            name, kms, alg = "stage", kt[1], K1 * (8 * 2 * Np * M + 160)
        else:
            i = int(np.argmax(kt[:3]))
            name, kms = ["volume", "face", "lift_update"][i], kt[i]
            alg = {"volume": K1 * (8 * Np * M * 2 + 8 * Nf * M + 32),
                   "face": (3 * K1 // 2) * 2 * (8 * s1.Ng * M) * 2 + (3 * K1 // 2) * 16,
                   "lift_update": K1 * (8 * Np * M * 3 + 8 * Nf * M + 8)}[name]
        ach = alg / (kms / 1000.0) / 1e9
        roofline = {"bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                    "frac": ach / peaks["hbm_gbs"], "traffic": profile_traffic().get(f"{prec}:{name}:{WORKLOAD}"),
                    "kernel": name, "peak_source": f"{peak_src} hbm_gbs",
                    "note": "dominant kernel of one rank's share, timed on a whole-mesh handle of that size"}
        s1.close()
    if rank == 0:
        nsend = sum(d.send_count)
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "mixed(tf32x3 tensor, fp32 acc, f64 state)",
            "data": "synthetic",
            "config": {"workload": f"euler_vortex_N4_K{K_local}_per_rank_partitioned", "K_global": mesh.K,
                       "K_rank0": K_local, "N": p.N, "fields": d.shape[2], "precision": prec,
                       "parallelism": f"halo x{world} (RCB strips, NCCL trace exchange per stage)",
                       "cut_faces_rank0": nsend,
                       "halo_bytes_per_stage_rank0": nsend * d.block_bytes[prec] * 2,
                       "l2_flush": "inputs larger than L2 (state + stage + scratch per rank > 126 MiB)"},
            "gpu_launches": args.steps * (26 if prec == "fp64" else 16), "clocks": clocks, "roofline": roofline,
            "e2e": e2e, "cpu_baseline": None, **extra,
        }
        print(json.dumps(line), flush=True)
    d.close()
    dist.barrier()
    dist.destroy_process_group()
    return 0


def e2e_pipelined(s, stream, U0, dt0, prec: str, ne: int) -> float:
    """Seconds for ne independent steps streamed through the public API with no
    host wait between steps: each step's input is uploaded from pinned host
    memory on an upload stream, handed to the handle (whose stream is
    ``stream``) by apollo_dg_set_state_async, stepped by apollo_dg_step_async,
    taken back by apollo_dg_get_state_async and downloaded to pinned host
    memory on a download stream; events order the three streams, two device
    buffers each way let the copies of neighbouring steps overlap the compute."""
    import torch
    shape = s.shape
    hU = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    hU.numpy()[...] = U0
    hO = [torch.empty(shape, dtype=torch.float64, pin_memory=True) for _ in range(2)]
    dU = [torch.empty(shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    dO = [torch.empty(shape, dtype=torch.float64, device="cuda") for _ in range(2)]
    up, down = torch.cuda.Stream(), torch.cuda.Stream()
    ev_up = [torch.cuda.Event() for _ in range(2)]       # input b uploaded
    ev_taken = [torch.cuda.Event() for _ in range(2)]    # input b copied into the handle
    ev_out = [torch.cuda.Event() for _ in range(2)]      # result b in dO[b]
    ev_down = [torch.cuda.Event() for _ in range(2)]     # result b downloaded

    def run(n):
        for b in range(2):
            ev_taken[b].record(stream)
            ev_down[b].record(down)
        for i in range(n):
            b = i % 2
            up.wait_event(ev_taken[b])
            with torch.cuda.stream(up):
                dU[b].copy_(hU, non_blocking=True)
                ev_up[b].record(up)
            stream.wait_event(ev_up[b])
            s.set_state_async(dU[b])
            ev_taken[b].record(stream)
            s.advance_async(1, 0.0, dt0, precision=prec)
            stream.wait_event(ev_down[b])
            s.get_state_async(dO[b])
            ev_out[b].record(stream)
            down.wait_event(ev_out[b])
            with torch.cuda.stream(down):
                hO[b].copy_(dO[b], non_blocking=True)
                ev_down[b].record(down)
        torch.cuda.synchronize()

    run(2)
    t0 = time.perf_counter()
    run(ne)
    el = time.perf_counter() - t0
    # every result is the one step of U0
    ref = s.get_state()
    assert np.array_equal(hO[(ne - 1) % 2].numpy(), ref)
    return el


def ours_arm(args):
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if (world > 1 and not args.replicas) or args.partitioned:
        return partitioned_arm(args, rank, world, local)
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist_mod.init_process_group("nccl", timeout=timedelta(seconds=120))
        dist = dist_mod
    from apollo_b200 import NodalDG2d, problems

    p = problems.euler_vortex(n=args.n, N=args.order, fields=4)
    stream = torch.cuda.Stream()
    s = NodalDG2d(p.N, p.cfl, p.equation, p.eq_params, p.mesh, device=local, stream=stream.cuda_stream)
    x, y = s.node_coords()
    U0 = np.ascontiguousarray(p.ic(x, y))
    s.set_state(U0)
    dt0 = s.init_dt()

    prec = args.precision
    if prec == "auto":
        prec = "fp64"
        try:
            s.step(0.0, 0.0, U0[:0] if False else U0, precision="mixed")
            prec = "mixed"
        except Exception:
            prec = "fp64"
    dofs = s.K * s.Np * s.m

    def timed(precision, steps, warmup):
        s.set_state(U0)
        s.advance_async(warmup, 0.0, dt0, precision=precision)
        t_w, dt_w = s.time()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            s.advance_async(steps, t_w, dt_w, precision=precision)
            e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist:
            tt = torch.tensor([ms], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = float(tt.item())
        return ms

    with ClockSampler(local) as clk:
        ms = timed(prec, args.steps, args.warmup)
    clocks = clk.summary()
    ms_step = ms / args.steps
    value = dofs * world * args.steps / (ms / 1000.0)
    t_end, _ = s.time()
    U_end = s.get_state()
    l2_exact = float(np.linalg.norm(U_end - p.exact(x, y, t_end)) / np.linalg.norm(p.exact(x, y, t_end)))

    extra = {}
    if prec == "mixed":
        ms64 = timed("fp64", args.steps, args.warmup)
        extra["fp64"] = {"value": dofs * world * args.steps / (ms64 / 1000.0), "ms_per_step": ms64 / args.steps}
        try:
            # the float64 stepper against the float64 pipe: Survey-8d contraction
            # FLOPs, 2 m (3 Nc Np + 2 Nf Np + Np^2) per element per stage
            Nc, Nf = s.Nc, 3 * s.Ng
            flops = 5 * s.K * 2 * s.m * (3 * Nc * s.Np + 2 * Nf * s.Np + s.Np * s.Np)
            ach = flops / (ms64 / args.steps / 1000.0) / 1e12
            pk = fp64_gemm_peak(local)
            extra["fp64"]["roofline"] = {"bound": "fp64", "achieved": ach, "peak": pk, "unit": "TFLOP/s",
                                         "frac": ach / pk, "flops_per_step": flops,
                                         "peak_source": "cuBLAS DGEMM 4096^3 on this GPU (torch.matmul, best of 5)"}
        except Exception as exc:
            extra["fp64"]["roofline"] = {"error": str(exc)}
        extra["speedup_vs_fp64"] = ms64 / ms
        if not args.no_l2_500:
            # the stated error: both forms over the configuration's 500 steps
            ends = {}
            for pr in ("fp64", "mixed"):
                s.set_state(U0)
                s.advance(500, 0.0, dt0, precision=pr)
                ends[pr] = s.get_state()
            extra["l2_mixed_vs_fp64_500_steps"] = float(np.linalg.norm(ends["mixed"] - ends["fp64"]) /
                                                         np.linalg.norm(ends["fp64"]))

    # per-kernel device time and the roofline of the dominant kernel
    s.set_state(U0)
    kt = s.kernel_times(10, precision=prec)
    peaks, peak_src = measured_peaks()
    N, K, M = p.N, s.K, s.m
    Np, Nc, Ng = s.Np, s.Nc, s.Ng
    Nf = 3 * Ng
    nfaces = 3 * K // 2
    if prec == "mixed":
        # one right-hand side = the trace kernel (state -> fp32 face traces) and
        # the fused stage kernel in right-hand-side mode
        names = ["traces", "stage", "unused"]
        alg_bytes = {  # compulsory bytes per launch
            "traces": K * (8 * Np * M + 4 * Nf * M),
            "stage": K * (8 * 2 * Np * M + 160),  # read x, write the RHS, geometry
        }
        alg_flops = {  # contraction flops (multiply-adds x2), pointwise flux excluded
            "traces": K * 2 * M * Nf * Np,
            "stage": K * 2 * M * (3 * Nc * Np + 2 * Nf * Np + Np * Np),
        }
        kt = kt[:2]
    else:
        names = ["volume", "face", "lift_update"]
        alg_bytes = {  # compulsory bytes per launch (float64)
            "volume": K * (8 * Np * M + 8 * Np * M + 8 * Nf * M + 32),
            "face": nfaces * 2 * (8 * Ng * M) * 2 + nfaces * 16,
            "lift_update": K * (8 * Np * M * 3 + 8 * Nf * M + 8),
        }
        alg_flops = {
            "volume": K * 2 * M * (Nc * Np + 2 * Nc * Np + Nf * Np),
            "face": nfaces * Ng * 60,
            "lift_update": K * 2 * M * Nf * Np,
        }
    dom = int(np.argmax(kt))
    dname = names[dom]
    achieved = alg_bytes[dname] / (kt[dom] / 1000.0) / 1e9
    traffic = profile_traffic().get(f"{prec}:{dname}:{workload_name(p.N, s.K)}")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "traffic": traffic, "kernel": dname,
                "peak_source": f"{peak_src} hbm_gbs",
                "kernel_ms": dict(zip(names, [float(v) for v in kt])),
                "contraction_tflops": alg_flops[dname] / (kt[dom] / 1000.0) / 1e12,
                "note": "float64 kernels are bounded by the FP64 pipe (B200 nominal 37 TFLOP/s), not HBM"}
    if prec == "mixed":
        roofline["note"] = ("stage kernel: tf32x3 tcgen05 contractions; bounded in practice by shared-memory "
                            "bandwidth and issue latency, not HBM (see profiles/)")
    # the whole stage (what one SSPRK stage must move at the least: read the
    # stage state and the step's initial state, write the new stage state, plus
    # 160 B of geometry per element), timed as a fifth of the measured step
    stage_b = 8 * 3 * Np * M + 160
    stage_ms = ms_step / 5.0
    stage_ach = stage_b * K / (stage_ms / 1000.0) / 1e9
    stage_traffic = (profile_traffic().get(f"mixed:stage:{workload_name(p.N, s.K)}") if prec == "mixed" else
                     sum(profile_traffic().get(f"fp64:{k}:{workload_name(p.N, s.K)}") or 0
                         for k in ("volume", "face", "lift_update")) or None)
    roofline["stage_mode"] = {"bytes_per_element": stage_b, "bytes": stage_b * K, "stage_ms": stage_ms,
                              "achieved": stage_ach, "frac": stage_ach / peaks["hbm_gbs"],
                              "traffic": stage_traffic,
                              "how": "compulsory bytes of one stage / (ms_per_step / 5); traffic: DRAM bytes of "
                                     "one stage from one-pass ncu captures at this mesh"}

    e2e = None
    if not args.no_e2e:
        # end to end through the public API: per step, the state from pinned host
        # memory to the device, one SSPRK step, the state back to pinned host memory
        hU = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
        hU.numpy()[...] = U0
        hO = torch.empty(s.shape, dtype=torch.float64, pin_memory=True)
        t, dt = 0.0, dt0
        ne = max(3, min(args.steps, 50))
        for _ in range(2):
            s.set_state(hU.numpy())
            t, dt = s.advance(1, t, dt, precision=prec)
            s.get_state(hO.numpy())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(ne):
            s.set_state(hU.numpy())
            t, dt = s.advance(1, t, dt, precision=prec)
            s.get_state(hO.numpy())
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        if dist:
            tt = torch.tensor([el], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        nb = s.K * s.Np * s.m * 8
        serial = dofs * world * ne / el
        el_p = e2e_pipelined(s, stream, U0, dt0, prec, ne)
        if dist:
            tt = torch.tensor([el_p], device="cuda")
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el_p = float(tt.item())
        e2e = {"value": dofs * world * ne / el_p, "unit": METRIC, "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb,
               "steps": ne, "serial_value": serial,
               "how": "wall clock over independent steps streamed through the public API with no host wait "
                      "between steps: each step's input copied from pinned host memory to a device buffer on an "
                      "upload stream, apollo_dg_set_state_async (device pointer), apollo_dg_step_async (1 step), "
                      "apollo_dg_get_state_async (device pointer), and the result copied to pinned host memory "
                      "on a download stream, events ordering the streams so that the copies of neighbouring "
                      "steps overlap the compute; serial_value: apollo_dg_set_state, apollo_dg_step and "
                      "apollo_dg_get_state with host pointers, one step at a time"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # Apollo's own code where it is built (oracle/_ref), on every host
        # core; the oracle's restatement on the benchmark mesh beside it
        try:
            port = cpu_sample()
        except Exception as exc:  # the CPU arm never hides a GPU result
            port = {"value": None, "error": str(exc)}
        try:
            ref = apollo_cpu_rate(steps=3, warmup=1)
        except Exception as exc:
            ref = None
            port["reference_error"] = str(exc)
        if ref is not None:
            cpu = {"value": ref["value"], "unit": METRIC, "cores": ref["cores"], "kind": "reference",
                   "sample": ref["sample"], "seconds": ref["seconds"]}
            extra["cpu_port"] = port
        else:
            cpu = port

    adj = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        try:
            adj = adjoint_measure(args, local)
        except Exception as exc:  # reported, never hides the headline
            adj = {"error": str(exc)}
    if adj is not None:
        extra["adjoint"] = adj
    if rank == 0 and world == 1 and not args.no_ensemble:
        try:
            extra["ensemble"] = ensemble_measure(args, local)
        except Exception as exc:  # reported, never hides the headline
            extra["ensemble"] = {"error": str(exc)}
    if rank == 0 and world == 1 and not args.no_configs:
        for key, fn in (("advection", advection_measure), ("maxwell_tm", maxwell_measure)):
            try:
                extra[key] = fn(args, local, cpu=not args.no_cpu_baseline)
            except Exception as exc:  # reported, never hides the headline
                extra[key] = {"error": str(exc)}
        if not args.no_cpu_baseline:
            try:
                extra["cpu_extra"] = cpu_extra(os.cpu_count() or 1)
            except Exception as exc:
                extra["cpu_extra"] = {"error": str(exc)}
            try:
                ref_extra = apollo_cpu_extra()
                if ref_extra is not None:
                    extra["apollo_cpu"] = ref_extra
            except Exception as exc:
                extra["apollo_cpu"] = {"error": str(exc)}

    if rank == 0:
        # our kernels per step: float64 5 x (volume, face, lift) + finalize;
        # mixed 5 fused stages + finalize (the trace kernel runs in the warm-up)
        line = {
            "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if prec == "fp64" else "mixed(tf32x3 tensor, fp32 acc, f64 state)",
            "data": "synthetic",
            "config": {"workload": workload_name(p.N, s.K), "K": s.K, "N": N, "Np": Np, "fields": M, "flux": "LF",
                       "cfl": p.cfl,
                       "precision": prec, "l2_flush": "inputs larger than L2 (state + stage + scratch "
                       f"{(dofs * 8 * 4 + 2 * K * Nf * M * 8) / 2**20:.0f} MiB > 126 MiB)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "l2_vs_exact_vortex": l2_exact, "t_end": t_end,
            "gpu_launches": args.steps * (16 if prec == "fp64" else 6), "clocks": clocks, "roofline": roofline, "e2e": e2e,
            "cpu_baseline": cpu, **extra,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.rhs_only:
        return rhs_only(args)
    if args.vjp_only:
        return vjp_only(args)
    if args.steps_only:
        return steps_only(args)
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
