"""Benchmark: time steps/s of the 3D lid-driven-cavity hex8 solve on B200.

One "step" is one time step of the solver (time update, boundary conditions,
Newton loop with assembly and Krylov solves to the absolute 1e-8 residual).
The default workload is the graded 115^3 hex8 cavity (1,520,875 elements,
1,560,896 nodes, 6.24 M dofs, Re = 1000, dt = 0.1, generalised-alpha
rho_inf = 0) with the reference's iterative option family: BiCGStab with a
block-Jacobi ILU preconditioner (one block, as a single process) at rtol
1e-10.  W warm-up steps from rest run first, then exactly K timed steps.

Arms:
  default          the CUDA library through its C ABI (device-resident state);
                   also an end-to-end number through the same API with the
                   state crossing host<->device every step.
  --impl reference the CPU restatement of the reference path (oracle/) on all
                   host cores, same workload, same solver options.

Multi-GPU (torchrun, N > 1): the path does not shard, every rank advances an
independent replica ("replicas only"); value = N*K / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "3D LDC hex8 time steps/s on 1 B200 (surrogate-guess vs plain) at 1e-8 residual"

# Solver presets (Handle keywords).  The default is the reference's BiCGStab
# option file (input/petsc_options_bcgs.dat) with one ILU(0) block;
# "gmres-pbjacobi" is the point-block Jacobi GMRES used before the ILU
# preconditioner existed (restart per workload).
SOLVERS = {
    "bcgs-ilu0": {"ksp": "bcgs", "pc": "bjacobi", "ilu_levels": 0, "rtol": 1e-10, "max_it": 10000},
    "bcgs-ilu1": {"ksp": "bcgs", "pc": "bjacobi", "ilu_levels": 1, "rtol": 1e-10, "max_it": 10000},
    "bcgs-ilu3": {"ksp": "bcgs", "pc": "bjacobi", "ilu_levels": 3, "rtol": 1e-10, "max_it": 10000},
    "gmres20-ilu1": {"ksp": "gmres", "restart": 20, "pc": "bjacobi", "ilu_levels": 1, "rtol": 1e-10,
                     "max_it": 10000},
    "gmres-pbjacobi": {"ksp": "gmres", "pc": "pbjacobi", "rtol": 1e-10, "max_it": 40000},
}
DEFAULT_SOLVER = "bcgs-ilu0"

WORKLOADS = {
    # name: (n per side, steps in the configuration, GMRES restart of the pbjacobi preset)
    "ldc3d_16": (16, 50, 400),
    "ldc3d_32": (32, 50, 400),
    "ldc3d_64": (64, 20, 800),
    "ldc3d_115": (115, 20, 1000),
    # O-grid around a cylinder, 256 x 128 quads (learned-guess configuration)
    "cylinder_wake": (256, 3000, 400),
}
DEFAULT_WORKLOAD = "ldc3d_115"
# solver preset when --solver is not given: the reference's BiCGStab option
# file (input/petsc_options_bcgs.dat) keeps its ILU(3) blocks on the 2D wake,
# where ILU(0) needs 7x the iterations; ILU(0) on the 3D cavities
WORKLOAD_SOLVER = {"cylinder_wake": "bcgs-ilu3"}

SMI_QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=4)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=list(WORKLOADS))
    p.add_argument("--solver", default=None, choices=list(SOLVERS),
                   help=f"solver preset (default {DEFAULT_SOLVER}; {WORKLOAD_SOLVER})")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-variant", action="store_true",
                   help="skip the mixed-precision + extrapolation-guess variant on the same time steps")
    p.add_argument("--precision", default="fp64", choices=["fp64", "mixed"],
                   help="mixed: FP64 flexible GMRES outer solves around FP32 BiCGStab inner solves with the FP32 "
                        "preconditioner")
    p.add_argument("--method", default="plain", choices=["plain", "surrogate", "extrapolation", "batch", "kernels"],
                   help="surrogate / extrapolation: run the plain solve for --train-steps, then time the "
                        "following steps from that state with mixed precision and the learned (surrogate) or "
                        "min-residual extrapolation initial guess; the line also carries every other variant "
                        "on the same steps from the same state, the plain FP64 path among them")
    p.add_argument("--train-steps", type=int, default=None,
                   help="plain steps before the evaluation window (default 20; 1000 on the wake, whose "
                        "configuration trains on steps 0-1000 and evaluates after them)")
    p.add_argument("--train-first", type=int, default=0,
                   help="first training sample n (u_{n-1}, u_n -> u_{n+1}); 0 = two steps after the lid ramp")
    p.add_argument("--train-iters", type=int, default=3000)
    p.add_argument("--newton-rtol", type=float, default=0.0,
                   help="surrogate/extrapolation: extra relative Newton test for the mixed-precision variants "
                        "(||F|| <= r ||F_0||, F_0 the constant predictor's iteration-0 residual); 0 = the 1e-8 "
                        "absolute test only")
    p.add_argument("--variants", default=None,
                   help="surrogate/extrapolation: comma-separated subset of " + ",".join(GUESS_VARIANTS) +
                        " (default: all on the 3D cavities, the FP64 ones on the 2D wake)")
    p.add_argument("--batch-count", type=int, default=64, help="batch: number of independent 2D cavities")
    p.add_argument("--kernel-restart", type=int, default=40,
                   help="kernels: GMRES restart of the bounded profiling case")
    p.add_argument("--kernel-its", type=int, default=40,
                   help="kernels: GMRES iterations of the bounded profiling case")
    p.add_argument("--kernel-net", action="store_true",
                   help="kernels: also one forward pass of the guess network (random weights) on the workload's mesh")
    p.add_argument("--no-batch-mixed", action="store_true", help="batch: skip the mixed-precision batch arm")
    p.add_argument("--no-batch-learned", action="store_true",
                   help="batch: skip the arm with the shared, Re-conditioned guess network")
    p.add_argument("--batch-schedule", default="auto",
                   help="batch: 'auto' (autotune during the warm-up steps) or 'C,K,D' (concurrency, chunk, depth)")
    a = p.parse_args()
    if a.solver is None:
        a.solver = WORKLOAD_SOLVER.get(a.workload, DEFAULT_SOLVER)
    if a.train_steps is None:
        a.train_steps = 1000 if a.workload == "cylinder_wake" else 20
    return a


def solver_options(name, solver=DEFAULT_SOLVER):
    opts = dict(SOLVERS[solver])
    if solver == "gmres-pbjacobi":
        opts["restart"] = WORKLOADS[name][2]
    return opts


def make_case(name, precision="fp64", solver=DEFAULT_SOLVER):
    from cfdsfemmpi_b200 import meshgen
    n, steps, _ = WORKLOADS[name]
    if name == "cylinder_wake":
        mesh, ctrl = meshgen.cylinder_ogrid(), meshgen.control_for(steps, 0.1, 0.01)
    else:
        mesh, ctrl, _ = meshgen.case_hex(n, steps, mu=0.001, dt=0.1)
    opts = solver_options(name, solver)
    if precision == "mixed":
        opts = mixed_options(opts)
    return mesh, ctrl, opts


def initial_state(name, mesh):
    """State at t = 0: rest, and on the wake the seeded transverse-velocity
    perturbation (uniform, amplitude 1e-3) that starts the shedding."""
    import numpy as np
    if name == "cylinder_wake":
        from cfdsfemmpi_b200 import meshgen
        return meshgen.cylinder_initial_state(mesh)
    return np.zeros(mesh.nNode * mesh.ndof)


def mixed_options(opts):
    """Mixed-precision solver with the preconditioner of `opts`: FP64 flexible
    GMRES(30) outer solves on the FP64 matrix to the step's Newton target,
    preconditioned by 20 FP32 BiCGStab iterations (inner rtol 1e-2) on an FP32
    copy with the FP32 form of the same preconditioner."""
    o = {k: v for k, v in opts.items() if k in ("pc", "ilu_levels", "bjacobi_blocks")}
    o.update(ksp="gmres", restart=30, rtol=1e-10, refine_rtol=1e-10, precision="mixed", inner_restart=20,
             inner_rtol=1e-2, max_it=2000)
    return o


# mixed-precision variants beside the plain line: the outer solve stopped at
# the Newton tolerance's scale (max(1e-10 ||b||, 1e-9): where the initial
# guess pays), or carried to a true residual of 1e-11 ||b|| (the accuracy of
# the plain path's solves)
MIXED_REGIMES = {"newton_floor": {}, "accurate": {"refine_rtol": 1e-11, "refine_atol": -1.0}}


def oracle_options(opts):
    """OracleFEM keywords for the same solver as the Handle keywords `opts`."""
    o = {"solver": opts.get("ksp", "gmres"), "rtol": opts["rtol"], "pc": opts["pc"],
         "max_it": opts.get("max_it", 10000)}
    if "restart" in opts:
        o["restart"] = opts["restart"]
    if opts["pc"] == "bjacobi":
        o["ilu_levels"] = opts.get("ilu_levels", 0)
        o["bjacobi_blocks"] = opts.get("bjacobi_blocks", 1)
    return o


def pc_label(opts):
    if opts["pc"] == "bjacobi":
        lev = opts.get("ilu_levels", 0)
        return f"block Jacobi, {opts.get('bjacobi_blocks', 1)} block(s) of " + ("LU" if lev < 0 else f"ILU({lev})")
    return opts["pc"]


def solver_label(opts):
    ksp = opts.get("ksp", "gmres")
    k = {"gmres": f"GMRES({opts.get('restart', 30)})", "bcgs": "BiCGStab", "preonly": "preonly"}[ksp]
    return f"{k} + {pc_label(opts)}, rtol {opts['rtol']:g}"


def workload_config(name, mesh, opts, extra=None):
    n = WORKLOADS[name][0]
    if name == "cylinder_wake":
        wl = (f"{name}: 2D cylinder wake, O-grid 256 x 128 quads ({mesh.nElem} elements, {mesh.nNode} nodes, "
              f"{mesh.nNode * 3} dofs), r 0.5..20, Re 100, dt 0.1, gen-alpha rho_inf 0, seeded 1e-3 transverse "
              "perturbation")
    else:
        wl = (f"{name}: graded-cube lid-driven cavity, {n}^3 hex8 ({mesh.nElem} elements, "
              f"{mesh.nNode} nodes, {mesh.nNode * 4} dofs), Re 1000, dt 0.1, gen-alpha rho_inf 0")
    cfg = {"workload": wl,
           "method": ("plain (reference-identical constant predictor), FP64" if opts.get("precision", "fp64") == "fp64"
                      else "plain predictor, mixed precision: FP64 flexible GMRES outer solves, FP32 BiCGStab + FP32 "
                           "preconditioner inner solves, FP64 Newton residual"),
           "solver": f"Newton to 1e-8 abs; {solver_label(opts)}",
           "l2": "flushed between timed steps (256 MiB write)"}
    if extra:
        cfg.update(extra)
    return cfg


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={SMI_QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier_max(world, value):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.barrier()
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


KINDS = ("spmv", "ortho", "elem_k", "elem_f", "trsv", "ilu", "bcgs")

# Work per timed step of the default workloads, as the GPU arm measures it on
# steps W+1..W+K with W = 3 (the same algorithm as the CPU restatement): Newton
# assemblies, linear solves, and Krylov iterations.  The reference arm scales
# its bounded per-step sample with these counts; the GPU arm's own
# cpu_baseline uses the live counts of its first timed step instead.
STEP_WORK = {
    ("ldc3d_115", "bcgs-ilu0"): (2, 1, 155),
    ("ldc3d_115", "bcgs-ilu1"): (2, 1, 97),
}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    from cfdsfemmpi_b200 import Handle

    torch.cuda.set_device(local)
    mesh, ctrl, opts = make_case(args.workload, args.precision, args.solver)
    h = Handle(mesh, ctrl, **opts)
    stream = torch.cuda.ExternalStream(h.stream_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    timeNow = ctrl.dt
    stats = []

    def one_step(record):
        nonlocal timeNow
        tf = timeNow if timeNow <= 1.0 else 1.0
        st = h.step(timeNow, tf).as_dict()
        timeNow = timeNow + ctrl.dt
        if record:
            stats.append(st)
        return st

    for _ in range(args.warmup):
        one_step(False)
    torch.cuda.synchronize()
    # state at the start of the timed window: the end-to-end replay and the
    # CPU sample start from it
    s0 = h.get_solution()
    p0, d0 = h.get_history()
    t_start = timeNow
    launches0 = h.launch_count()
    sampler = ClockSampler(local)
    sampler.start()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    total_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        one_step(True)
        e1.record(stream)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    launches = h.launch_count() - launches0
    t_max = barrier_max(world, total_ms)
    value = world * args.steps / (t_max * 1e-3)
    s_final = h.get_solution()

    # end to end through the C ABI with host buffers: the same K time steps
    # replayed on the same handle from the saved state; every step copies the
    # state in from pinned host memory, steps, and copies the result back
    # (cfdgpu_set_solution + cfdgpu_step + cfdgpu_get_solution)
    e2e = None
    if not args.no_e2e:
        n = h.n
        pin = torch.empty(n, dtype=torch.float64, pin_memory=True)
        pin.numpy()[:] = s0
        h.set_history(p0, d0)
        t2 = t_start
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            h.set_solution_ptr(pin.data_ptr())
            h.step(t2, t2 if t2 <= 1.0 else 1.0)
            t2 = t2 + ctrl.dt
            h.get_solution_ptr(pin.data_ptr())
        dt_e2e = time.perf_counter() - t0
        dt_e2e = barrier_max(world, dt_e2e)
        e2e = {"value": world * args.steps / dt_e2e, "unit": "steps/s", "steps": args.steps,
               "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n,
               "replay_bitwise_equal": bool(np.array_equal(pin.numpy(), s_final)),
               "api": "cfdgpu_set_solution + cfdgpu_step + cfdgpu_get_solution (pinned host buffers), the same "
                      "time steps as the device-resident timing replayed from the same state, host wall clock"}

    # dominant kernel: profile one more step with per-launch CUDA events
    h.set_profiling(True)
    one_step(False)
    kinds = {k: h.kernel_stats(k) for k in KINDS}
    h.set_profiling(False)
    prof_total = sum(v[1] for v in kinds.values())
    dom = max(kinds, key=lambda k: kinds[k][1])
    nl, ms, by = kinds[dom]
    peak, peak_src = _hbm_peak()
    achieved = (by / nl) / (ms / nl * 1e-3) / 1e9 if nl else None
    # DRAM traffic per launch: the ratio of ncu-measured DRAM bytes to
    # algorithmic bytes for this kernel kind and workload (profiles/), times
    # this run's algorithmic bytes per launch
    traffic = None
    tpath = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tpath) and nl:
        try:
            ent = json.load(open(tpath)).get(f"{args.workload}/{args.solver}", {}).get(dom)
            if ent:
                traffic = ent["dram_bytes_per_algorithmic_byte"] * by / nl
        except Exception:
            traffic = None
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_source": peak_src,
                "unit": "GB/s", "frac": (achieved / peak) if achieved else None, "traffic": traffic,
                "algorithmic_bytes_per_launch": by / nl if nl else None,
                "avg_launch_ms": ms / nl if nl else None, "launches_profiled": nl,
                "share_of_profiled_step": ms / prof_total if prof_total else None,
                "kernels": {k: {"launches": v[0], "ms": round(v[1], 4),
                                "gbs": (v[2] / (v[1] * 1e-3) / 1e9) if v[1] else None} for k, v in kinds.items()}}

    # the mixed-precision + min-residual extrapolation-guess variants, on K
    # time steps from the same state as a plain FP64 run of the same steps,
    # with their field errors against it.  The guess extrapolates the last
    # increment u_n - u_{n-1}; while the lid velocity ramps up (t <= 1) the
    # iteration-0 residual is dominated by the lid's own change, which no
    # combination of interior increments removes, so a window inside the ramp
    # is moved to the first steps whose u_n and u_{n-1} both carry the full
    # lid velocity (the plain run continues there untimed, then times the
    # window the same way as above).
    variant = None
    if not args.no_variant and args.precision == "fp64":
        t_guess = 1.0 + 2 * ctrl.dt
        if t_start >= t_guess - 1e-9:
            vs0, vp0, vd0, vt, v_final, v_ms, v_its = s0, p0, d0, t_start, s_final, total_ms, its_of(stats)
        else:
            while timeNow < t_guess - 1e-9:
                one_step(False)
            torch.cuda.synchronize()
            vs0 = h.get_solution()
            vp0, vd0 = h.get_history()
            vt = timeNow
            v_ms, v_stats = 0.0, []
            for _ in range(args.steps):
                with torch.cuda.stream(stream):
                    flush.fill_(1)
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                v_stats.append(one_step(False))
                e1.record(stream)
                e1.synchronize()
                v_ms += e0.elapsed_time(e1)
            v_final = h.get_solution()
            v_its = its_of(v_stats)
        k0 = int(round(vt / ctrl.dt))
        # the same window solved tighter (FP64, rtol 1e-12): how far the
        # plain path's own rtol-1e-10 answer is determined
        s_tight = run_fixed(mesh, ctrl, dict(opts, rtol=1e-12), vs0, vp0, vd0, vt, args.steps)
        refs = {"plain_fp64": v_final, "fp64_rtol1e-12": s_tight}
        variant = {"window": f"steps {k0}..{k0 + args.steps - 1} (t = {vt:.1f}..{vt + (args.steps - 1) * ctrl.dt:.1f}"
                             "; the lid at full velocity)",
                   "plain_fp64": {"value": args.steps / (v_ms * 1e-3), "unit": "steps/s",
                                  "ms_per_step": v_ms / args.steps, "krylov_iters": v_its,
                                  "field_error_vs_fp64_rtol1e-12": field_errors(v_final, s_tight, mesh.ndof)}}
        for name, extra in MIXED_REGIMES.items():
            variant[name] = run_variant(args, mesh, ctrl, dict(mixed_options(opts), **extra), vs0, vp0, vd0, vt,
                                        refs, v_ms, flush)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        st0 = stats[0]
        work = (st0["newton_iters"], len(st0["ksp_its"]), sum(st0["ksp_its"]))
        cpu = cpu_baseline_sample(args, mesh, ctrl, opts, s0, d0, t_start, work)
    h.close()
    its = its_of(stats)
    newt = [s["newton_iters"] for s in stats]
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
            "data": "synthetic: graded-cube hex8 cavity generated in-process (no dataset)",
            "config": workload_config(args.workload, mesh, opts,
                                      {"parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                                       "timed_steps": f"{args.warmup + 1}..{args.warmup + args.steps} of the run"}),
            "newton_iters_per_step": statistics.mean(newt) if newt else None,
            "krylov_iters_per_step": statistics.mean(its) if its else None,
            "krylov_iters": its,
            "all_converged": all(s["converged"] for s in stats),
            "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "mixed_guess_variant": variant, "clocks": clocks}
    return line


def its_of(stats):
    """Krylov iterations of each time step (summed over its Newton solves)."""
    return [sum(s["ksp_its"]) for s in stats]


def field_errors(a, b, ndof):
    """Relative L2 differences of the whole state, the velocity and the
    pressure; "pressure_mod_constant" compares the pressures after removing
    each one's mean (the pressure's constant mode is fixed only through the
    single pinned node, so every solver leaves it determined to the size of
    its final residual divided by a tiny eigenvalue)."""
    import numpy as np
    a = a.reshape(-1, ndof)
    b = b.reshape(-1, ndof)
    rel = lambda x, y: float(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-300))
    pa, pb = a[:, -1] - a[:, -1].mean(), b[:, -1] - b[:, -1].mean()
    return {"all": rel(a, b), "velocity": rel(a[:, :-1], b[:, :-1]), "pressure": rel(a[:, -1], b[:, -1]),
            "pressure_mod_constant": rel(pa, pb)}


def run_fixed(mesh, ctrl, kw, s0, p0, d0, t_start, steps):
    """`steps` untimed time steps with solver keywords `kw` from a saved
    state; returns the final state."""
    from cfdsfemmpi_b200 import Handle
    h = Handle(mesh, ctrl, **kw)
    h.set_solution(s0)
    h.set_history(p0, d0)
    t = t_start
    for _ in range(steps):
        h.step(t, t if t <= 1.0 else 1.0)
        t = t + ctrl.dt
    sol = h.get_solution()
    h.close()
    return sol


def run_variant(args, mesh, ctrl, kw, s0, p0, d0, t_start, refs, plain_ms, flush):
    """Mixed precision (FP64 flexible GMRES around FP32 BiCGStab with the FP32
    preconditioner, solver keywords `kw`) with the min-residual extrapolation
    initial guess, on the timed steps of the plain run from the same state;
    device-timed like the plain run."""
    import statistics as stat
    import torch
    from cfdsfemmpi_b200 import Handle
    h = Handle(mesh, ctrl, guess="extrapolation", **kw)
    h.set_solution(s0)
    h.set_history(p0, d0)
    stream = torch.cuda.ExternalStream(h.stream_ptr())
    t = t_start
    total, st = 0.0, []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.fill_(1)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st.append(h.step(t, t if t <= 1.0 else 1.0).as_dict())
        e1.record(stream)
        e1.synchronize()
        total += e0.elapsed_time(e1)
        t = t + ctrl.dt
    sol = h.get_solution()
    h.close()
    floor = kw.get("refine_atol", 0.0)
    floor_s = "1e-9 (Newton tolerance / 10)" if floor == 0.0 else ("none" if floor < 0 else f"{floor:g}")
    return {"method": "mixed precision + min-residual extrapolation initial guess",
            "solver": f"outer FGMRES({kw['restart']}) on the FP64 matrix to max({kw['refine_rtol']:g} ||b||, "
                      f"floor {floor_s}); preconditioner {kw['inner_restart']} FP32 BiCGStab its (rtol "
                      f"{kw['inner_rtol']:g}) with FP32 {pc_label(kw)}",
            "value": args.steps / (total * 1e-3), "unit": "steps/s", "ms_per_step": total / args.steps,
            "speedup_vs_plain": plain_ms / total,
            "outer_iters_per_step": stat.mean(sum(s["ksp_its"]) for s in st),
            "newton_iters_per_step": stat.mean(s["newton_iters"] for s in st),
            "guess_residual_ratio": stat.mean(s["guess_norm"] / s["plain_norm"] if s["plain_norm"] > 0 else 1.0
                                              for s in st),
            "all_converged": all(s["converged"] for s in st),
            "final_residuals": [s["norms"][-1] for s in st],
            **{f"field_error_vs_{k}": field_errors(sol, v, mesh.ndof) for k, v in refs.items()}}


def _cpu_sample_once(fem, ctrl, state, t_start, nits):
    """Bounded sample of one time step on the host: the step's iteration-0
    assembly, the preconditioner set-up (ILU factorisation, timed on its
    second run so that first-touch page faults of the factor arrays are not
    counted) and the cost of one Krylov iteration, taken as the difference of
    solves of 2 nits and nits iterations (set-up and start-up cancel).
    Returns (t_assembly, t_setup, t_per_it, its)."""
    import oracle
    s0, d0 = state
    fem.soln = s0.copy()
    fem.solnDot = d0.copy()
    fem.timeNow = t_start
    fem.td = oracle.time_params(ctrl.tis, ctrl.rhoInf, ctrl.dt)
    fem.time_update()
    tf = t_start if t_start <= 1.0 else 1.0
    fem.solnApplied[fem.dbc_index] = fem.dbc_value * tf - fem.soln[fem.dbc_index]
    fem.update_iter_step()
    t0 = time.perf_counter()
    fem.assemble(0)
    t_asm = time.perf_counter() - t0
    t_fac = 0.0
    if fem.pc == 3:
        fem.factor_ilu()
        t0 = time.perf_counter()
        fem.factor_ilu()
        t_fac = time.perf_counter() - t0
    rhs = fem.rhs.copy()
    times, its = [], []
    for k in (nits, 2 * nits):
        fem.rhs[:] = rhs
        fem.max_it = k
        t0 = time.perf_counter()
        _, info = fem.linear_solve()
        times.append(time.perf_counter() - t0)
        its.append(info["its"])
    dits = max(1, its[1] - its[0])
    return t_asm, t_fac, max(0.0, times[1] - times[0]) / dits, its[1]


def cpu_baseline_sample(args, mesh, ctrl, opts, s0, d0, t_start, work, nits=None):
    """CPU restatement of the reference path (oracle/, OpenMP on all host
    threads, the same solver) on a bounded sample of the first timed step,
    scaled to a full step with that step's Newton/Krylov counts (the reference
    reassembles the tangent every Newton iteration and sets the
    preconditioner up for every solve)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    threads = os.cpu_count() or 1
    fem = oracle.OracleFEM(mesh, ctrl, **oracle_options(opts), threads=threads)
    nits = nits or (5 if fem.solver == "bcgs" else opts.get("restart", 20))
    t_asm, t_fac, t_it, its_done = _cpu_sample_once(fem, ctrl, (s0, d0), t_start, nits)
    n_asm, n_solve, n_its = work
    t_step = n_asm * t_asm + n_solve * t_fac + n_its * t_it
    return {"value": 1.0 / t_step, "unit": "steps/s", "cores": threads, "kind": "port",
            "sample": f"time step t = {t_start:.1f} of the same run from the GPU state: iteration-0 assembly "
                      f"{t_asm:.2f} s, preconditioner set-up {t_fac:.2f} s, Krylov iteration {t_it:.3f} s (difference "
                      f"of {nits}- and {2 * nits}-iteration solves); scaled to the step's {n_asm} assemblies, "
                      f"{n_solve} set-ups and {n_its} Krylov iterations = {t_step:.1f} s",
            "t_assembly_s": t_asm, "t_setup_s": t_fac, "t_krylov_it_s": t_it}


def run_reference(args, world, rank):
    """CPU restatement of the reference path, all host threads.  Workloads up
    to 64^3 run whole time steps; at 115^3 every step is a bounded sample
    (assembly, preconditioner set-up and a few Krylov iterations of the
    configuration's time step from rest) scaled with the measured work per
    step of the same solver (STEP_WORK)."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import numpy as np
    import oracle
    mesh, ctrl, opts = make_case(args.workload, args.precision, args.solver)
    threads = os.cpu_count() or 1
    fem = oracle.OracleFEM(mesh, ctrl, **oracle_options(opts), threads=threads)
    bounded = (args.workload, args.solver) in STEP_WORK
    base = {"metric": METRIC, "unit": "steps/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "impl": "reference",
            "data": "synthetic: graded-cube hex8 cavity generated in-process (no dataset)",
            "config": workload_config(args.workload, mesh, opts, {"parallelism": "host cores"})}
    if bounded:
        n_asm, n_solve, n_its = STEP_WORK[(args.workload, args.solver)]
        zero = np.zeros(mesh.nNode * mesh.ndof)
        samples = []
        for k in range(args.warmup + args.steps):
            r = _cpu_sample_once(fem, ctrl, (zero, zero), ctrl.dt, 5 if fem.solver == "bcgs" else 20)
            if k >= args.warmup:
                samples.append(r)
        t_asm = statistics.mean(r[0] for r in samples)
        t_fac = statistics.mean(r[1] for r in samples)
        t_it = statistics.mean(r[2] for r in samples)
        t_step = n_asm * t_asm + n_solve * t_fac + n_its * t_it
        value = 1.0 / t_step
        sample = (f"bounded sample per step (the first time step's iteration-0 assembly, ILU set-up and one "
                  f"Krylov iteration from the difference of 5- and 10-iteration solves; {args.steps} timed repeats "
                  f"after {args.warmup}), scaled to "
                  f"{n_asm} assemblies, {n_solve} set-ups and {n_its} Krylov iterations per step (the work the GPU "
                  f"arm measures per timed step with the same solver): {t_step:.1f} s per step")
        line = dict(base, value=value, ms_per_step=t_step * 1e3,
                    cpu_baseline={"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
                                  "sample": sample, "t_assembly_s": t_asm, "t_setup_s": t_fac, "t_krylov_it_s": t_it},
                    e2e={"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        return line

    def one():
        fem.step()
        fem.timeNow = fem.timeNow + ctrl.dt

    for _ in range(args.warmup):
        one()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one()
    dt = time.perf_counter() - t0
    stats = fem.stats[args.warmup:]
    value = args.steps / dt
    return dict(base, value=value, ms_per_step=dt * 1e3 / args.steps,
                krylov_iters_per_step=statistics.mean(sum(s["gmres_its"]) for s in stats),
                cpu_baseline={"value": value, "unit": "steps/s", "cores": threads, "kind": "port",
                              "sample": f"time steps {args.warmup + 1}..{args.warmup + args.steps} of the run, "
                                        "C restatement (OpenMP) of the reference path"},
                e2e={"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})


GUESS_VARIANTS = {
    # name: (precision, guess)
    "plain": ("fp64", None),
    "fp64_extrapolation": ("fp64", "extrapolation"),
    "mixed": ("mixed", None),
    "mixed_extrapolation": ("mixed", "extrapolation"),
    "mixed_learned": ("mixed", ("network", "extrapolation")),
    "fp64_learned": ("fp64", ("network", "extrapolation")),
    "reference_tight": ("fp64", None),
}
DEFAULT_VARIANTS = {"cylinder_wake": ("plain", "fp64_extrapolation", "fp64_learned", "reference_tight")}


def run_guess(args, world, rank, local):
    """Initial-guess variants on the same held-out steps from the same state
    (the plain solver's state after --train-steps steps): constant predictor
    (the reference's), min-residual extrapolation and the learned guess, in
    FP64 and in mixed precision.  The headline is the variant --method names;
    every variant's throughput, iteration counts and field error against an
    FP64 rtol-1e-12 run are reported beside it."""
    import numpy as np
    import torch
    from cfdsfemmpi_b200 import Handle
    from cfdsfemmpi_b200._lib import Mpnn
    from cfdsfemmpi_b200.surrogate import fit_scales, train_guess

    torch.cuda.set_device(local)
    mesh, ctrl, opts = make_case(args.workload, solver=args.solver)
    ramp_end = int(round(1.0 / ctrl.dt))          # the Dirichlet data ramp up to t = 1
    first = args.train_first or ramp_end + 2
    if args.variants:
        names = [v for v in args.variants.split(",") if v]
        bad = [v for v in names if v not in GUESS_VARIANTS]
        if bad:
            raise SystemExit(f"unknown variants {bad}")
    else:
        names = list(DEFAULT_VARIANTS.get(args.workload, [k for k in GUESS_VARIANTS if k != "fp64_learned"]))
    head_name = ("mixed_learned" if args.method == "surrogate" else "mixed_extrapolation")
    if head_name not in names:
        head_name = head_name.replace("mixed_", "fp64_")
    for need in (head_name, "plain", "reference_tight"):
        if need not in names:
            names.append(need)
    T0 = time.perf_counter()
    h0 = Handle(mesh, ctrl, **opts)
    u0 = initial_state(args.workload, mesh)
    h0.set_solution(u0)
    traj = [u0]
    t = ctrl.dt
    for _ in range(args.train_steps):
        h0.step(t, t if t <= 1.0 else 1.0)
        traj.append(h0.get_solution())
        t = t + ctrl.dt
    prev0, dot0 = h0.get_history()
    h0.close()
    t_traj = time.perf_counter() - T0
    results = {}
    trained = None
    for name in names:
        prec, guess = GUESS_VARIANTS[name]
        kw = dict(opts)
        if prec == "mixed":
            kw = mixed_options(opts)
            if args.newton_rtol > 0:
                kw.update(newton_rtol=args.newton_rtol, newton_max_iter=30)
        if name == "reference_tight":
            kw.update(rtol=1e-12, max_it=40000)
        h = Handle(mesh, ctrl, **kw)
        h.set_solution(traj[-1])
        h.set_history(prev0, dot0)
        net = None
        t_train = 0.0
        if guess == "extrapolation":
            h.set_guess_mode(("extrapolation",))
        elif guess is not None:
            if trained is None:
                T1 = time.perf_counter()
                net, losses = train_guess(h, traj, iters=args.train_iters, lr=2e-3, seed=0, first=first)
                torch.cuda.synchronize()
                t_train = time.perf_counter() - T1
                trained = (net.get_params(), fit_scales(traj, mesh.ndof), losses)
            else:
                # the same trained network on this variant's handle
                net = Mpnn(h, seed=0)
                net.set_scales(*trained[1])
                net.set_params(trained[0])
            net.attach(guess)
        stream = torch.cuda.ExternalStream(h.stream_ptr())
        tt = t
        for _ in range(args.warmup):
            h.step(tt, tt if tt <= 1.0 else 1.0)
            tt = tt + ctrl.dt
        total_ms, stats = 0.0, []
        for _ in range(args.steps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            stats.append(h.step(tt, tt if tt <= 1.0 else 1.0).as_dict())
            e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
            tt = tt + ctrl.dt
        results[name] = {"ms": total_ms, "stats": stats, "soln": h.get_solution(), "t_train": t_train}
        if net is not None:
            net.close()
        h.close()
    ref = results["reference_tight"]["soln"].reshape(-1, mesh.ndof)

    def err(sol):
        d = sol.reshape(-1, mesh.ndof) - ref
        return {"all": float(np.linalg.norm(d) / np.linalg.norm(ref)),
                "velocity": float(np.linalg.norm(d[:, :-1]) / np.linalg.norm(ref[:, :-1])),
                "pressure": float(np.linalg.norm(d[:, -1]) / np.linalg.norm(ref[:, -1]))}

    def summary(r):
        st = r["stats"]
        return {"value": args.steps / (r["ms"] * 1e-3), "unit": "steps/s",
                "gmres_iters_per_step": statistics.mean(sum(s["ksp_its"]) for s in st),
                "newton_iters_per_step": statistics.mean(s["newton_iters"] for s in st),
                "guess_used_steps": sum(s["guess_used"] for s in st),
                "guess_residual_ratio": statistics.mean(s["guess_norm"] / s["plain_norm"] if s["plain_norm"] > 0
                                                        else 1.0 for s in st),
                "all_converged": all(s["converged"] for s in st),
                "field_error_vs_fp64_rtol1e-12": err(r["soln"])}

    head, pl = results[head_name], results["plain"]
    t_max = barrier_max(world, head["ms"])
    value = world * args.steps / (t_max * 1e-3)
    t0 = args.train_steps + args.warmup + 1
    method = ("learned initial guess (3-layer 64-wide message passing, BF16 tensor-core kernels, trained on "
              f"samples {first}..{args.train_steps - 1} of the plain solve to predict the correction over linear "
              "extrapolation; combined with the extrapolated increment by the exact min-residual coefficients)"
              if args.method == "surrogate" else
              "min-residual extrapolation initial guess (u_n + a (u_n - u_{n-1}), a minimising the affine "
              "iteration-0 residual)") + \
        (" + mixed precision (FP64 flexible GMRES around FP32 BiCGStab with the FP32 preconditioner)"
         if head_name.startswith("mixed") else ", FP64")
    line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if head_name.startswith("mixed") else "f64", "impl": "ours",
            "method": head_name,
            "data": "synthetic: graded-cube hex8 cavity generated in-process (no dataset)",
            "config": workload_config(args.workload, mesh, opts, {
                "method": method,
                "timed_steps": f"{t0}..{t0 + args.steps - 1} (after the training window)",
                "l2": "not flushed (inputs resident, same protocol for every variant here)"}),
            "speedup_vs_plain": pl["ms"] / head["ms"],
            "variants_same_steps": {k: summary(v) for k, v in results.items()},
            "train_seconds": max(r["t_train"] for r in results.values()), "trajectory_seconds": t_traj}
    return line


# GMRES(50)+Jacobi at rtol 1e-10 (the 2D configuration) stalls on the larger
# batch cavities (n >= 129 reach max_it); GMRES(400) + point-block Jacobi at
# rtol 1e-8 converges every step in two Newton iterations
def _hbm_peak():
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(peaks["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


BATCH_SOLVER = {"restart": 400, "rtol": 1e-8, "pc": "pbjacobi", "max_it": 20000}


def run_batch(args, world, rank, local):
    """Many independent 2D cavities (uneven sizes and Reynolds numbers) on one
    GPU: the batch runtime (concurrent instances, autotuned schedule) against
    the same instances stepped one by one through their own handles, on the
    same time steps.  Both arms end each instance step in a stream
    synchronisation, so host wall clock brackets the device work."""
    import numpy as np
    import torch
    from cfdsfemmpi_b200 import Batch, Handle, meshgen

    torch.cuda.set_device(local)
    cases = meshgen.batch_cases(count=args.batch_count, seed=2024 + rank)
    pairs = [(m, c) for m, c, _, _ in cases]
    dt = pairs[0][1].dt
    ntune = 12        # autotuner candidates: concurrency (32, all) x chunk (4, 8) x depth (1, 2, 4)
    warm = max(args.warmup, ntune)
    steps = args.steps
    n = len(pairs)

    def times(k):
        return np.full(n, dt * (k + 1))

    # one by one: each instance's own handle, instances in turn every step
    hs = [Handle(m, c, **BATCH_SOLVER) for m, c in pairs]
    for k in range(warm):
        for i, h in enumerate(hs):
            t = float(times(k)[i])
            h.step(t, min(t, 1.0))
    torch.cuda.synchronize()
    lat_seq, its_seq = [], 0
    lat_mat = np.zeros((steps, n))
    T0 = time.perf_counter()
    for k in range(warm, warm + steps):
        for i, h in enumerate(hs):
            t = float(times(k)[i])
            t1 = time.perf_counter()
            st = h.step(t, min(t, 1.0))
            lat_seq.append((time.perf_counter() - t1) * 1e3)
            lat_mat[k - warm, i] = lat_seq[-1]
            its_seq += sum(st.ksp_its[:st.newton_iters])
    torch.cuda.synchronize()
    wall_seq = time.perf_counter() - T0
    sol_seq = [h.get_solution() for h in hs]
    for h in hs:
        h.close()
    del hs

    # batch
    b = Batch(pairs, **BATCH_SOLVER)
    if args.batch_schedule == "auto":
        b.set_schedule(0, 0)
    else:
        c, ch, dp = (int(x) for x in args.batch_schedule.split(","))
        b.set_schedule(c, ch, dp)
    for k in range(warm):
        b.step(times(k))
    sched = b.schedule()
    torch.cuda.synchronize()
    launches0 = sum(h.launch_count() for h in b.handles)
    clocks = ClockSampler(local)
    clocks.start()
    # algorithmic HBM bytes of the Krylov work (the whole step's dominant
    # cost): per Arnoldi step j of a cycle, SpMV with the point-block Jacobi
    # epilogue B*b^2*8 + 4B + 4(N+1) + 2V + N*b^2*8 and Gram-Schmidt (2j+5)V
    infos = [h.pattern_info() for h in b.handles]
    m = BATCH_SOLVER["restart"]

    def krylov_bytes(i, its):
        pi = infos[i]
        bb = pi.ndof * pi.ndof
        V = 8.0 * pi.nNode * pi.ndof
        spmv = pi.nnzb * bb * 8 + 4 * pi.nnzb + 4 * (pi.nNode + 1) + 2 * V + pi.nNode * bb * 8
        full, rest = divmod(its, m)
        js = full * (m * (m - 1)) + rest * (rest - 1)          # 2 * sum of j over the iterations
        return its * spmv + (js + 5 * its) * V

    lat_b, its_b, alg_bytes = [], 0, 0.0
    T0 = time.perf_counter()
    for k in range(warm, warm + steps):
        st, lat = b.step(times(k))
        lat_b.extend(lat.tolist())
        its_b += sum(sum(s.ksp_its[:s.newton_iters]) for s in st)
        for i, s_ in enumerate(st):
            for q in range(s_.newton_iters):
                alg_bytes += krylov_bytes(i, s_.ksp_its[q])
    torch.cuda.synchronize()
    wall_b = time.perf_counter() - T0
    ck = clocks.stop()
    sol_b = [h.get_solution() for h in b.handles]
    launches = sum(h.launch_count() for h in b.handles) - launches0
    b.close()
    equal = sum(int(np.array_equal(a, c)) for a, c in zip(sol_b, sol_seq))

    # the same batch with the min-residual extrapolation guess (FP64)
    bx = Batch(pairs, guess="extrapolation", **BATCH_SOLVER)
    bx.set_schedule(0, 0, 0)
    for k in range(warm):
        bx.step(times(k))
    torch.cuda.synchronize()
    T0 = time.perf_counter()
    lat_x, its_x = [], 0
    for k in range(warm, warm + steps):
        st, lat = bx.step(times(k))
        lat_x.extend(lat.tolist())
        its_x += sum(sum(s.ksp_its[:s.newton_iters]) for s in st)
    torch.cuda.synchronize()
    wall_x = time.perf_counter() - T0
    sol_x = [h.get_solution() for h in bx.handles]
    bx.close()
    dvx = []
    for a, c in zip(sol_x, sol_b):
        a3, c3 = a.reshape(-1, 3), c.reshape(-1, 3)
        dvx.append(float(np.linalg.norm(a3[:, :2] - c3[:, :2]) / max(np.linalg.norm(c3[:, :2]), 1e-300)))
    extrap = {"value": n * steps / wall_x, "unit": "instance-steps/s", "speedup_vs_one_by_one": wall_seq / wall_x,
              "latency_ms": {"p50": float(np.percentile(lat_x, 50)), "p99": float(np.percentile(lat_x, 99))},
              "gmres_iters": int(its_x), "max_velocity_rel_diff_vs_constant_predictor": max(dvx)}

    # the same batch with one guess network shared by every instance and
    # conditioned on its Reynolds number (input channel log Re / log 5000):
    # trained on the warm-up steps' samples of all instances (each on its own
    # mesh), then each instance's network (the shared weights, its own
    # condition) combined with the extrapolated increment by the min-residual
    # rule, on the same timed steps
    learned = None
    if not args.no_batch_learned:
        from cfdsfemmpi_b200.surrogate import attach_shared, train_shared
        bl = Batch(pairs, **BATCH_SOLVER)
        bl.set_schedule(0, 0, 0)
        trajs = [[h.get_solution()] for h in bl.handles]
        for k in range(warm):
            bl.step(times(k))
            for i, h in enumerate(bl.handles):
                trajs[i].append(h.get_solution())
        conds = [float(np.log(re) / np.log(5000.0)) for _, _, _, re in cases]
        torch.cuda.synchronize()
        T1 = time.perf_counter()
        net0, shared, losses = train_shared(bl.handles, trajs, conds, iters=args.train_iters, lr=2e-3, seed=0,
                                            first=2)
        torch.cuda.synchronize()
        t_train = time.perf_counter() - T1
        nsamples = net0.num_samples
        net0.close()
        nets = [attach_shared(h, shared, c) for h, c in zip(bl.handles, conds)]
        del trajs
        torch.cuda.synchronize()
        T0 = time.perf_counter()
        lat_l, its_l, used, ratios = [], 0, 0, []
        for k in range(warm, warm + steps):
            st, lat = bl.step(times(k))
            lat_l.extend(lat.tolist())
            its_l += sum(sum(s.ksp_its[:s.newton_iters]) for s in st)
            for s_ in st:
                used += int(s_.guess_used)
                ratios.append(s_.guess_norm / s_.plain_norm if s_.plain_norm > 0 else 1.0)
        torch.cuda.synchronize()
        wall_l = time.perf_counter() - T0
        sol_l = [h.get_solution() for h in bl.handles]
        for q in nets:
            q.close()
        bl.close()
        dvl = []
        for a, c in zip(sol_l, sol_b):
            a3, c3 = a.reshape(-1, 3), c.reshape(-1, 3)
            dvl.append(float(np.linalg.norm(a3[:, :2] - c3[:, :2]) / max(np.linalg.norm(c3[:, :2]), 1e-300)))
        learned = {"value": n * steps / wall_l, "unit": "instance-steps/s", "speedup_vs_one_by_one": wall_seq / wall_l,
                   "latency_ms": {"p50": float(np.percentile(lat_l, 50)), "p99": float(np.percentile(lat_l, 99))},
                   "gmres_iters": int(its_l), "guess_used": f"{used}/{n * steps}",
                   "guess_residual_ratio_mean": float(np.mean(ratios)),
                   "training": {"samples": int(nsamples), "iters": args.train_iters, "seconds": t_train,
                                "loss_first_last": [float(losses[0]), float(losses[-1])],
                                "samples_from": f"steps 2..{warm - 1} of every instance"},
                   "max_velocity_rel_diff_vs_constant_predictor": max(dvl)}

    # the same batch in mixed precision (FP64 flexible GMRES around FP32 BiCGStab,
    # FP64 refinement and Newton residual), same steps and schedule rule
    mixed = None
    if not args.no_batch_mixed:
        bm = Batch(pairs, **dict(BATCH_SOLVER, restart=30, precision="mixed", inner_restart=20, inner_rtol=1e-2,
                                 max_it=2000))
        bm.set_schedule(0, 0, 0)
        for k in range(warm):
            bm.step(times(k))
        torch.cuda.synchronize()
        T0 = time.perf_counter()
        lat_m = []
        for k in range(warm, warm + steps):
            st, lat = bm.step(times(k))
            lat_m.extend(lat.tolist())
        torch.cuda.synchronize()
        wall_m = time.perf_counter() - T0
        sol_m = [h.get_solution() for h in bm.handles]
        sched_m = bm.schedule()
        bm.close()
        dv = []
        for a, c in zip(sol_m, sol_b):
            a3, c3 = a.reshape(-1, 3), c.reshape(-1, 3)
            dv.append(float(np.linalg.norm(a3[:, :2] - c3[:, :2]) / max(np.linalg.norm(c3[:, :2]), 1e-300)))
        mixed = {"value": n * steps / wall_m, "unit": "instance-steps/s", "speedup_vs_one_by_one": wall_seq / wall_m,
                 "latency_ms": {"p50": float(np.percentile(lat_m, 50)), "p99": float(np.percentile(lat_m, 99))},
                 "schedule": sched_m, "max_velocity_rel_diff_vs_fp64_batch": max(dv)}
    wall_max = barrier_max(world, wall_b)
    value = world * n * steps / wall_max
    dofs = sum(m.nNode * m.ndof for m, _ in pairs)
    line = {"metric": "2D LDC batch: instance time steps/s on 1 B200 (64 cavities, uneven n and Re) at 1e-8 residual",
            "value": value, "unit": "instance-steps/s", "n_gpus": world, "steps": steps, "warmup": warm,
            "ms_per_step": wall_max * 1e3 / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "impl": "ours", "method": "batch",
            "data": "synthetic: 2D quad4 cavities generated in-process (n ~ U{24..160}, log Re ~ U[log 100, log 5000], "
                    "seed 2024, dt 0.05)",
            "config": {"workload": f"batch of {n} 2D lid-driven cavities, {dofs} dofs in total",
                       "solver": "Newton to 1e-8 abs; GMRES(400) + point-block Jacobi, rtol 1e-8",
                       "schedule": sched, "timing": "host wall clock; every instance step ends in a stream "
                       "synchronisation", "l2": "inputs resident; no flush (the batch is the working set)",
                       "timed_steps": f"{warm + 1}..{warm + steps}", "parallelism": "single GPU, concurrent streams"},
            "latency_ms": {"p50": float(np.percentile(lat_b, 50)), "p99": float(np.percentile(lat_b, 99))},
            "roofline": {"bound": "hbm", "kernel": "all Krylov kernels of all instances (SpMV + Gram-Schmidt)",
                         "achieved": alg_bytes / wall_b / 1e9, "peak": _hbm_peak()[0], "peak_source": _hbm_peak()[1],
                         "unit": "GB/s", "frac": alg_bytes / wall_b / 1e9 / _hbm_peak()[0], "traffic": None,
                         "algorithmic_bytes_per_step": alg_bytes / steps,
                         "one_by_one_achieved": alg_bytes / wall_seq / 1e9},
            "one_by_one": {"value": n * steps / wall_seq, "unit": "instance-steps/s",
                           "latency_ms": {"p50": float(np.percentile(lat_seq, 50)),
                                          "p99": float(np.percentile(lat_seq, 99))},
                           "gmres_iters": int(its_seq)},
            "speedup_vs_one_by_one": wall_seq / wall_b, "gmres_iters": int(its_b),
            # no schedule can finish a batch step before its slowest instance
            # finishes alone: the longest single-instance step time bounds it
            "critical_path_ms": {"slowest_instance_alone_per_step": float(lat_mat.max(axis=1).mean()),
                                 "instance": int(lat_mat.sum(axis=0).argmax()),
                                 "n": int(cases[int(lat_mat.sum(axis=0).argmax())][2]),
                                 "Re": float(cases[int(lat_mat.sum(axis=0).argmax())][3]),
                                 "batch_step_over_bound": float(wall_b * 1e3 / steps / lat_mat.max(axis=1).mean())},
            "instances_bitwise_equal_to_one_by_one": f"{equal}/{n}", "gpu_launches": int(launches),
            "extrapolation_guess_batch": extrap,
            "shared_learned_guess_batch": learned,
            "mixed_precision_batch": mixed,
            "clocks": ck}
    return line


def run_kernels(args, local):
    """A bounded case for profiling the hot kernels in isolation: the
    workload's mesh, one tangent assembly (iteration-0 semantics) on a seeded
    random state, and exactly --kernel-its GMRES iterations with restart
    --kernel-restart on a seeded right-hand side, so a profiler sees the
    element kernels, the BSR SpMV with its preconditioner and the Gram-Schmidt
    kernels at realistic sizes and the run ends by itself.  Prints one JSON
    line (not a benchmark value)."""
    import numpy as np
    import torch
    from cfdsfemmpi_b200 import Handle, meshgen

    torch.cuda.set_device(local)
    n_side = WORKLOADS[args.workload][0]
    mesh, ctrl, _ = meshgen.case_hex(n_side, 2)
    kw = dict(solver_options(args.workload, args.solver), restart=args.kernel_restart, rtol=1e-30,
              max_it=args.kernel_its)
    h = Handle(mesh, ctrl, **kw)
    rng = np.random.default_rng(0)
    n = mesh.nNode * mesh.ndof
    prev = 0.1 * rng.standard_normal(n)
    h.set_element_state(prev, prev, np.zeros(n))
    t0 = time.perf_counter()
    h.assemble_export(0, want_values=False)
    b = rng.standard_normal(n)
    b[h.export_pattern()["fixed_dofs"]] = 0.0
    x, its, reason = h.solve_export(b)
    if args.kernel_net:
        from cfdsfemmpi_b200._lib import Mpnn
        net = Mpnn(h, seed=0)
        net.predict(prev, 0.5 * prev)
        net.close()
    dt = time.perf_counter() - t0
    line = {"method": "kernels", "workload": args.workload, "nodes": mesh.nNode, "solver": solver_label(kw),
            "restart": args.kernel_restart, "its": its, "reason": reason, "seconds": dt,
            "launches": h.launch_count(), "network_forward": bool(args.kernel_net)}
    h.close()
    return line


def main():
    args = parse()
    if args.impl == "reference":
        # host-only arm: rank 0 runs it, other ranks have nothing to do
        rank = int(os.environ.get("RANK", "0"))
        line = run_reference(args, int(os.environ.get("WORLD_SIZE", "1")), rank)
        if line is not None:
            print(json.dumps(line))
        return
    if args.method == "batch":
        # separate hardware queues for the instances' streams (read when the
        # CUDA context is created)
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    world, rank, local = dist_setup(args)
    if args.method == "kernels":
        line = run_kernels(args, local)
    elif args.method == "batch":
        line = run_batch(args, world, rank, local)
    elif args.method in ("surrogate", "extrapolation"):
        line = run_guess(args, world, rank, local)
    else:
        line = run_ours(args, world, rank, local)
    if rank == 0 and line is not None:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
