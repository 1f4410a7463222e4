"""Benchmark: SIMP iterations/s of the GMG-PCG minimum-compliance loop at 12.8M DOF.

Workload (the reference's large 3-D demo size): hex8 cantilever 256x128x128
(4,194,304 elements, 12,830,211 DOF), E0=1, Emin(void)=1e-9, nu=0.3, p=3, vf=0.1,
r_min=2, x=0 face clamped, unit total downward load on the bottom edge at x=L,
6-grid GMG (n_level=5, coarsest 675 DOF, FP64 Cholesky), PCG rtol 1e-6, move 0.2.
A step = one SIMP iteration (OC update + filter + SIMP law + GMG-PCG solve + compliance
+ sensitivity + filter transpose), warm-started like the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision fp64|mixed]
  python bench.py --impl reference ...   (CPU reference arm: the reference's CPU SIMP
                                           iteration, oracle/cpu_simp.py, on the host cores)

Prints one JSON line (rank 0).  `value` is device-timed with inputs resident in HBM;
`e2e` runs the same steps through the public API with the design kept in pinned host
memory (H2D of rho, D2H of rho_new and the compliance every step).  Every working array
(12.8M-DOF vectors, 1 GB level-1 operator) is larger than the 126 MB L2, so no flush is
needed between steps.
"""
import argparse
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "SIMP iter/s at 12.8M DOF: mixed-prec vs FP64 GMG-PCG, compl rel.err≤1e-6"
CONFIGS = {
    "cantilever_256x128x128": dict(nel=(256, 128, 128), vf=0.1, rmin=2.0, n_level=5, tol=1e-6),
    "cantilever_128x64x64": dict(nel=(128, 64, 64), vf=0.1, rmin=2.0, n_level=4, tol=1e-6),
    "cantilever_64x32x32": dict(nel=(64, 32, 32), vf=0.12, rmin=1.5, n_level=4, tol=1e-6),
}
# rtol of the FP64 oracle trajectory (nearly exact solves) the timed paths are compared with
ORACLE_RTOL = 1e-10
# PCG iterations of the CPU reference timed per step (the timed samples of oracle/cpu_simp.py)
CPU_PCG_SAMPLES = 8


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profile(config):
    """Per-launch DRAM bytes of the fine operator from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "fine_operator_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p)).get(config)
        return None if d is None else d.get("dram_bytes_per_launch")
    except Exception:
        return None


class ClockSampler:
    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"edge_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # nvidia-smi's start-up (NVML initialisation) must not overlap the timed region:
        # wait for its first sample (at most 10 s)
        import time
        t0 = time.time()
        while time.time() - t0 < 10.0 and self.proc.poll() is None:
            if os.path.exists(self.path) and os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) >= 8:
                try:
                    rows.append((float(f[0]), float(f[1]), f[4], f[5], f[6], f[7]))
                except ValueError:
                    pass
        if not rows:
            return None
        import statistics
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[2:]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        loaded = [r[0] for r in rows]
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(r[1] for r in rows), "reasons": sorted(reasons),
                "samples": len(rows)}


def build_problem(cfg, precision, n_smooth=3, graph=True, maxiter=1000):
    import numpy as np
    import torch
    import edge_to_b200 as eb
    nel = cfg["nel"]
    mesh = eb.CuStructuredMesh3D(*nel, *[float(v) for v in nel], stiffness=lambda x: eb.auto_stiffness(x, 1.0, 0.3))
    mat = eb.SingleMaterial(E=1.0, nu=0.3, void=1e-9, penalty=3.0, volume_fraction=cfg["vf"])
    k = eb.CuStructuredStiffnessKernel(mesh)
    filt = eb.CuStructuredFilter3D(mesh, cfg["rmin"])
    solver = eb.CuMultiGrid(mesh, k, tol=cfg["tol"], n_level=cfg["n_level"], maxiter=maxiter, precision=precision,
                            n_smooth=n_smooth, graph=graph)
    opt = eb.CuTopOpt(mesh, mat, k, solver, filt, max_iter=1, move=0.2, verbose=False)
    nx, ny, nz = nel[0] + 1, nel[1] + 1, nel[2] + 1
    j, k_ = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    face = (j * nx * nz + k_).ravel()                    # i = 0
    opt.add_BC_nodal(face, np.array([[True, True, True]]))
    edge = (0 * nx * nz + nel[0] * nz + np.arange(nz))    # i = nelx, j = 0
    opt.add_F_nodal(edge, np.array([[0.0, -1.0, 0.0]]) / edge.shape[0])
    rho = torch.full((mesh.n_elements,), cfg["vf"], dtype=torch.float64, device="cuda")
    return opt, rho


def timed_steps(opt, rho, dr, it, steps, ws, local, profile=True):
    """`steps` SIMP iterations between barriers + synchronisation, CUDA events on the
    library's stream (torch's current stream); returns the max-over-ranks time."""
    import ctypes
    import torch
    from edge_to_b200 import _lib
    stream = torch.cuda.current_stream()
    h = opt.kernel.handle
    pcg, comps = [], []
    clocks = ClockSampler(local)
    clocks.start()
    _barrier(ws)
    torch.cuda.synchronize()
    if profile:
        _lib.call("edge_profile_begin", h, 200000)
    n_before = ctypes.c_longlong()
    _lib.call("edge_launch_count", h, ctypes.byref(n_before))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    torch.cuda.nvtx.range_push("edge_timed")      # lets ncu --nvtx-include select the timed launches
    c = None
    for _ in range(steps):
        if profile:  # per-launch events: the OC update and the host-driven solve as separate calls
            rho = opt.update_design(rho, dr)
            c, dr, res = opt.solve_and_process(rho, it)
        else:        # one graph launch per SIMP iteration
            rho, c, dr, res = opt.iterate(rho, dr, it)
        pcg.append(opt.last_stats.get("pcg_iters", 0))
        comps.append(float(c))  # already on the host: the analysis returns it from a host read
        it += 1
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    _barrier(ws)
    n_after = ctypes.c_longlong()
    _lib.call("edge_launch_count", h, ctypes.byref(n_after))
    prof = None
    if profile:
        kms, kby, kl, tl = ctypes.c_double(), ctypes.c_double(), ctypes.c_int(), ctypes.c_longlong()
        _lib.call("edge_profile_end", h, ctypes.byref(kms), ctypes.byref(kby), ctypes.byref(kl), ctypes.byref(tl))
        prof = dict(kernel_ms=kms.value, kernel_bytes=kby.value, kernel_launches=kl.value)
    clk = clocks.stop()
    t_ms = _max_over_ranks(e0.elapsed_time(e1), ws)
    return dict(rho=rho, dr=dr, it=it, t_ms=t_ms, pcg=pcg, compliance=float(c), comps=comps, prof=prof, clocks=clk,
                launches=n_after.value - n_before.value)


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(v, ws):
    """The maximum of v over the ranks (a CUDA tensor under NCCL, a host tensor under gloo)."""
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    tt = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def _gather_over_ranks(v, ws):
    """The list of every rank's value v (rank order); [v] on one rank."""
    if ws == 1:
        return [v]
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    mine = torch.tensor([float(v)], dtype=torch.float64, device=dev)
    out = [torch.zeros_like(mine) for _ in range(ws)]
    dist.all_gather(out, mine)
    return [float(t.item()) for t in out]


def whole_job_rate(units_per_rank, ws, t_max_ms):
    """Units processed by all ranks per second, over the slowest rank's time: every rank does
    the same amount of work (replicas or equal shards), so the job ends with the slowest."""
    return ws * units_per_rank / (t_max_ms / 1e3)


def warm(opt, rho, warmup, comps=None):
    """Initial analysis + `warmup` untimed SIMP iterations (compliances appended to comps)."""
    c, dr, res = opt.solve_and_process(rho, 0)
    if comps is not None:
        comps.append(float(c))
    it = 0
    for _ in range(warmup):
        rho, c, dr, res = opt.iterate(rho, dr, it)
        if comps is not None:
            comps.append(float(c))
        it += 1
    return rho, dr, it


def trajectory_diff(comps_a, comps_b, rho_a, rho_b):
    """Per-iteration relative compliance difference of two SIMP trajectories from the same
    start, and the largest absolute difference of their designs after the last one."""
    d = [abs(a - b) / abs(b) for a, b in zip(comps_a, comps_b)]
    return {"iterations": len(d), "compliance_rel_diff_max": max(d) if d else None,
            "compliance_rel_diff_last": d[-1] if d else None,
            "rho_max_abs_diff_last": float((rho_a - rho_b).abs().max()),
            "compliance_rel_diff_per_iteration": [float(f"{v:.3e}") for v in d]}


def run_ours(args, cfg_name):
    import numpy as np
    import torch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    cfg = CONFIGS[cfg_name]
    cpu_job = None
    if ws == 1 and not args.no_cpu_baseline:
        cpu_job = start_cpu_reference(cfg_name, CPU_PCG_SAMPLES, max(1, (os.cpu_count() or 2) - 2))
    opt, rho = build_problem(cfg, args.precision, args.n_smooth, graph=not args.no_graph)
    if args.sweeps:
        from edge_to_b200 import _lib as _l
        pat = [int(v) for v in args.sweeps.split(",")]
        opt.solver.tune_sweeps = False
        opt.solver.sweeps = {"per_level": pat, "fixed": True}
        _l.call("edge_mg_set_sweeps", opt.kernel.handle, _l.int_array(pat), len(pat))
    if args.coarse_fp32:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_coarse_bf16", opt.kernel.handle, 0)
    if args.residual64:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_residual32", opt.kernel.handle, 0)
    if args.pdl:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_pdl", opt.kernel.handle, 1)
    if args.no_fuse:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_fuse", opt.kernel.handle, 0)
    if args.omega_schedule:
        opt.solver.mixed_omega = None
    if args.fuse_xr:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_fuse_xr", opt.kernel.handle, 1)
    if args.no_kind_tune:
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_kind_tune", opt.kernel.handle, 0)
    if args.galerkin == "direct":
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_galerkin_axis", opt.kernel.handle, 0)
    if args.stencil != "default":
        from edge_to_b200 import _lib as _l
        _l.call("edge_set_stencil_tiled", opt.kernel.handle, -1 if args.stencil == "linear" else 200000)
    traj = []
    rho, dr, it = warm(opt, rho, args.warmup, traj)
    # the state the timed steps start from; the end-to-end steps restart from it, so both
    # measure the same SIMP iterations (later iterations need more PCG iterations)
    start = (rho.clone(), dr.clone(), it, opt.solver.last_x0.clone() if opt.solver.last_x0 is not None else None)

    # ---------------- device-timed region: inputs resident in HBM; each solve is one CUDA
    # graph launch (per-launch events cannot sit inside a graph, so none are recorded here)
    m = timed_steps(opt, rho, dr, it, args.steps, ws, local, profile=False)
    rho, dr, it, t_ms = m["rho"], m["dr"], m["it"], m["t_ms"]
    traj += m["comps"]
    rho_traj = rho.detach().clone()
    # the state after the timed steps (the profiled step below continues from it)
    after = (rho.clone(), dr.clone(), it, opt.solver.last_x0.clone())
    # ---------------- end-to-end: design on the host, copies inside the timed region, from the
    # timed steps' starting state
    stream = torch.cuda.current_stream()
    rho0, dr_e, it_e, x0 = start
    if x0 is not None:
        opt.solver.last_x0.copy_(x0)
    rho_h = torch.empty(rho0.numel(), dtype=torch.float64, pin_memory=True)
    rho_h.copy_(rho0.cpu())
    out_h = torch.empty_like(rho_h)
    e2e_pcg = []
    _barrier(ws)
    torch.cuda.synchronize()
    s0 = torch.cuda.Event(enable_timing=True)
    s1 = torch.cuda.Event(enable_timing=True)
    s0.record(stream)
    for _ in range(args.steps):
        rho_d = rho_h.to("cuda", non_blocking=True)
        rho_n, c, dr_e, res = opt.iterate(rho_d, dr_e, it_e)
        out_h.copy_(rho_n, non_blocking=True)
        comp_host = float(c)  # D2H of the compliance (synchronising)
        e2e_pcg.append(opt.last_stats.get("pcg_iters", 0))
        rho_h, out_h = out_h, rho_h
        it_e += 1
    s1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = _max_over_ranks(s0.elapsed_time(s1), ws)
    # ---------------- back to the state after the timed steps
    rho, dr, it = after[0], after[1], after[2]
    opt.solver.last_x0.copy_(after[3])
    # ---------------- one more step with CUDA events around every fine-operator launch (the
    # host-driven loop, same launches) for the live roofline of the dominant kernel
    pm = timed_steps(opt, rho, dr, it, 1, ws, local, profile=True)
    rho, dr, it, prof = pm["rho"], pm["dr"], pm["it"], pm["prof"]
    # checked against a tight FP64 solve below: compliance, displacement and sensitivities
    rho_chk, c_chk = rho.detach().clone(), pm["compliance"]
    u_chk, dr_chk = opt.solver.last_x0.detach().clone(), dr.detach().clone().reshape(-1)

    bd = breakdown(opt, rho, dr, it) if args.breakdown else None
    tuned = opt.solver.tuned
    sweeps = opt.solver.sweeps
    fixed_omega = opt.solver.fixed_omega
    del opt, rho, dr, rho_h, out_h

    # ---------------- the plain FP64 path on the same workload, same steps (the metric's
    # denominator), when the timed path is the mixed-precision one
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64_compare:
        torch.cuda.empty_cache()
        opt64, rho64 = build_problem(cfg, "fp64")
        traj64 = []
        rho64, dr64, it64 = warm(opt64, rho64, args.warmup, traj64)
        f = timed_steps(opt64, rho64, dr64, it64, args.steps, ws, local, profile=False)
        traj64 += f["comps"]
        fp64 = {"value": whole_job_rate(args.steps, ws, f["t_ms"]), "ms_per_step": f["t_ms"] / args.steps,
                "pcg_iters_per_step": f["pcg"], "compliance_last": f["compliance"]}
        # the two SIMP trajectories (initial analysis, warm-up and timed iterations) from the
        # same start design, iteration by iteration
        fp64["trajectory"] = trajectory_diff(traj, traj64, rho_traj, f["rho"])
        # accuracy of each path against an rtol-1e-10 FP64 solve of the same design (its own
        # last design), outside every timed region
        opt64.solver.tol, opt64.solver.maxiter = 1e-10, 4000
        c_t64 = float(opt64.solve_and_process(f["rho"], f["it"])[0])
        c_tmx, dr_t, _ = opt64.solve_and_process(rho_chk, f["it"])
        c_tmx = float(c_tmx)
        u_t = opt64.solver.last_x0
        dr_t = dr_t.reshape(-1)
        fp64["compliance_rel_err_vs_tight_fp64"] = abs(f["compliance"] - c_t64) / abs(c_t64)
        fp64["mixed_vs_tight"] = {
            "compliance": abs(c_chk - c_tmx) / abs(c_tmx),
            "displacement": float(torch.linalg.norm(u_chk - u_t) / torch.linalg.norm(u_t)),
            "dc": float((dr_chk - dr_t).abs().max() / dr_t.abs().max())}
        rho64_last = f["rho"].detach().clone()
        del opt64, rho64, dr64, f
        if not args.no_oracle_trajectory:
            # the FP64 oracle trajectory: the same SIMP iterations with every solve at rtol
            # ORACLE_RTOL (nearly exact), against which both timed paths' compliances and
            # designs are compared iteration by iteration (outside every timed region)
            torch.cuda.empty_cache()
            opt_t, rho_t = build_problem(dict(cfg, tol=ORACLE_RTOL), "fp64", maxiter=5000)
            traj_t = []
            rho_t, _, _ = warm(opt_t, rho_t, args.warmup + args.steps, traj_t)
            fp64["oracle"] = {"rtol": ORACLE_RTOL,
                              "mixed": trajectory_diff(traj, traj_t, rho_traj, rho_t),
                              "fp64": trajectory_diff(traj64, traj_t, rho64_last, rho_t)}
            del opt_t, rho_t
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return None
    n_el = int(np.prod(cfg["nel"]))
    peak, peak_kind = peaks()
    kms, kby = prof["kernel_ms"], prof["kernel_bytes"]
    achieved = (kby / prof["kernel_launches"]) / (kms / prof["kernel_launches"] / 1e3) / 1e9 if kms > 0 else None
    traffic = traffic_from_profile(cfg_name)
    value = whole_job_rate(args.steps, ws, t_ms)
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "iter/s",
        "n_gpus": ws,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": t_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if args.precision == "fp64" else "f32+bf16/f64",
        "data": "synthetic: reference cantilever BCs and load, rho0 = vf, random-free",
        "config": {"workload": cfg_name, "dof": 3 * int(np.prod([n + 1 for n in cfg["nel"]])), "elements": n_el,
                   "n_level": cfg["n_level"], "rtol": cfg["tol"], "precision": args.precision,
                   "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
                   "l2": "working set > 126 MB L2 (no flush needed)",
                   "pcg_iters_per_step": m["pcg"], "compliance_last": m["compliance"],
                   "fine_tile": tuned, "sweeps": sweeps,
                   "coarse_stencils": "fp32" if (args.coarse_fp32 or args.precision == "fp64") else "bf16",
                   "residual_recurrence": "fp64" if (args.residual64 or args.precision == "fp64") else "fp32",
                   "level_stencil_kernel": args.stencil,
                   "galerkin_products": args.galerkin,
                   "programmatic_dependent_launch": args.pdl and not args.no_graph,
                   "fused_fine_launches": args.precision == "mixed" and not args.no_fuse,
                   "fused_xr_update": (args.precision == "mixed" and not args.no_fuse and args.fuse_xr
                                       and fixed_omega is not None),
                   "smoother_omega": (f"fixed at {fixed_omega}" if fixed_omega is not None
                                      else "reference schedule (0.40-0.45 on the fine level)")},
        "roofline": {"bound": "hbm", "kernel": "fine-level operator (k_fine3_cube/_pk/_tma + fused epilogues)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None, "peak_source": peak_kind,
                     "traffic": traffic, "traffic_case": "ncu DRAM bytes per launch, mean over the three fused "
                     "fine launches of one PCG iteration (profiles/fine_operator_traffic.json)" if traffic else None, "launches": prof["kernel_launches"], "kernel_ms": kms,
                     "algorithmic_bytes_per_launch": kby / max(1, prof["kernel_launches"]),
                     "share_of_step": kms / pm["t_ms"] if pm["t_ms"] else None,
                     "timing": "CUDA events around every fine-operator launch of one SIMP step run right "
                               "after the timed steps (host-driven PCG loop, same kernels and tiles)"},
        "e2e": {"value": whole_job_rate(args.steps, ws, e2e_ms), "unit": "iter/s", "h2d_bytes_per_step": 8 * n_el,
                "d2h_bytes_per_step": 8 * n_el + 8, "pcg_iters_per_step": e2e_pcg,
                "note": "the same SIMP iterations as the device-timed steps (restarted from their state)"},
        "gpu_launches": m["launches"],
        "matvecs": {"fine_per_s_kernel": prof["kernel_launches"] / (kms / 1e3) if kms > 0 else None,
                    "fine_per_step": prof["kernel_launches"],
                    "note": "fine-level operator applications (any epilogue); per_s_kernel = launches / their "
                            "CUDA-event time in the profiled step"},
        "clocks": m["clocks"],
    }
    if fp64 is not None:
        line["trajectory_vs_fp64"] = fp64.pop("trajectory")
        if "oracle" in fp64:
            line["trajectory_vs_fp64_oracle"] = fp64.pop("oracle")
        line["fp64_path"] = fp64
        line["mixed_over_fp64"] = value / fp64["value"]
        line["compliance_rel_err_vs_fp64"] = abs(m["compliance"] - fp64["compliance_last"]) / abs(
            fp64["compliance_last"])
        acc = fp64.pop("mixed_vs_tight")
        line["compliance_rel_err_vs_tight_fp64"] = acc["compliance"]
        line["accuracy_vs_tight_fp64"] = dict(acc, note="the timed path's last design solved again in FP64 at "
                                                      "rtol 1e-10: relative errors (displacement 2-norm, dc max-norm)")
    if bd is not None:
        line["breakdown_ms_per_step"] = bd
    if cpu_job is not None:
        line["cpu_baseline"] = cpu_reference_line(finish_cpu_reference(cpu_job, 900.0))
        line["cpu_baseline"]["note"] = ("run in a spawned process beside the GPU measurement on all host threads "
                                        "but two")
    return line


CATS = ["other", "fine_operator", "coarse_stencils", "transfers", "vector_pcg", "setup_galerkin_chol",
        "coarsest_solve", "oc_update", "filter_sensitivity"]


def breakdown(opt, rho, dr, it):
    """One more SIMP step (outside the timed region) with CUDA events around every launch."""
    import ctypes
    from edge_to_b200 import _lib
    h = opt.kernel.handle
    _lib.call("edge_breakdown_begin", h, 60000)
    rho = opt.update_design(rho, dr)
    opt.solve_and_process(rho, it)
    ms = (ctypes.c_double * 16)()
    nn = (ctypes.c_int * 16)()
    _lib.call("edge_breakdown_end", h, ms, nn, 16)
    return {CATS[i]: {"ms": round(ms[i], 3), "launches": nn[i]} for i in range(len(CATS))}


def _cpu_reference_worker(cfg_name, samples, threads, q):
    """Child process: the reference's CPU SIMP iteration (oracle/cpu_simp.py) timed on
    `threads` host threads; puts its measurement dict on q."""
    os.environ["NUMBA_NUM_THREADS"] = str(threads)
    try:
        from oracle import cpu_simp
        cfg = CONFIGS[cfg_name]
        q.put(cpu_simp.measure(cfg["nel"], cfg["vf"], cfg["rmin"], cfg["n_level"], cfg["tol"], samples=samples))
    except Exception as e:  # reported, not raised: the GPU measurement stands on its own
        q.put({"error": repr(e)})


def start_cpu_reference(cfg_name, samples, threads):
    """Starts the CPU reference measurement in a spawned process (before any GPU call, so
    the child holds no CUDA state), to run beside the GPU measurement."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    proc = ctx.Process(target=_cpu_reference_worker, args=(cfg_name, samples, threads, q), daemon=True)
    proc.start()
    return proc, q


def finish_cpu_reference(handle, timeout_s):
    proc, q = handle
    import queue
    try:
        m = q.get(timeout=timeout_s)
    except queue.Empty:
        m = {"error": f"no result within {timeout_s:.0f} s"}
    proc.join(timeout=10)
    if proc.is_alive():
        proc.kill()
    return m


def cpu_reference_line(m):
    """cpu_baseline object of the JSON line from a cpu_simp.measure result."""
    if "error" in m:
        return {"value": None, "unit": "iter/s", "cores": None, "kind": "port", "sample": m["error"]}
    return {"value": 1.0 / m["seconds_per_iteration"], "unit": "iter/s", "cores": m["threads"], "kind": "port",
            "sample": (f"the reference's CPU SIMP iteration (oracle/cpu_simp.py) on {m['threads']} threads: first "
                       f"analysis solved to rtol ({m['first_solve_pcg_iters']} PCG iterations, the CPU solver's own "
                       f"count; {m['first_solve_pcg_s']:.1f} s) with set-up {m['setup_s']:.2f} s, post "
                       f"{m['post_s']:.2f} s, OC {m['oc_s']:.2f} s, then {len(m['pcg_iteration_samples_s'])} more "
                       f"PCG iterations timed one by one (median {m['pcg_iteration_s']:.3f} s); iteration = set-up "
                       f"+ post + OC + {m['first_solve_pcg_iters']} x median = {m['seconds_per_iteration']:.1f} s. "
                       "Later SIMP iterations need more PCG iterations than this cold first solve, so the CPU "
                       f"rate is an upper bound. Fine product {m['matvec_s']:.3f} s (index arithmetic; "
                       f"{m['matvec_list_indexing_s']:.3f} s with the reference's element-list lookups)"),
            "detail": m}


def run_matvec(args, cfg_name):
    """Profiling helper: K fine-operator applications (kernel.dot) on the workload's grid,
    E = (0.1 + 0.9 * uniform)^3, x=0 face constrained.  Prints its own JSON line."""
    import numpy as np
    import torch
    opt, rho = build_problem(CONFIGS[cfg_name], args.precision)
    k = opt.kernel
    g = torch.Generator(device="cuda").manual_seed(0)
    E = (0.1 + 0.9 * torch.rand(k.n_elements, generator=g, device="cuda", dtype=torch.float64)) ** 3
    k.set_rho(E)
    u = torch.randn(k.shape[0], generator=g, device="cuda", dtype=torch.float64)
    from edge_to_b200 import _lib
    out = torch.empty_like(u)
    if args.tile is not None:
        _lib.call("edge_set_fine_tile", k.handle, args.tile, args.tile_bps)

    def apply():
        if args.precision == "fp64":
            k.dot(u)
        else:
            _lib.call("edge_matvec_f32", k.handle, _lib.ptr(u), _lib.ptr(out))
    for _ in range(args.warmup):
        apply()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        apply()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    n_dof, n_el = k.shape[0], k.n_elements
    w = 8 if args.precision == "fp64" else 4
    alg = 2 * w * n_dof + w * n_el
    peak, kind = peaks()
    return {"mode": "matvec", "workload": cfg_name, "tile": args.tile, "ms_per_matvec": ms, "algorithmic_bytes": alg,
            "GBps": alg / (ms / 1e3) / 1e9, "frac_of_peak": alg / (ms / 1e3) / 1e9 / peak, "peak_source": kind,
            "note": "includes the user-layout <-> slot-layout conversions of edge_matvec"}


def run_tiles(args, cfg_name):
    """Profiling helper: device time of every fine-kernel tile variant (plain product and
    smoother sweep, CUDA events around `steps` launches) on the workload's grid after one
    SIMP analysis, so E, the boundary conditions and the multigrid are the live ones."""
    import ctypes
    import torch
    from edge_to_b200 import _lib
    opt, rho = build_problem(CONFIGS[cfg_name], args.precision)
    h = opt.kernel.handle
    if args.tile is None:
        opt.solve_and_process(rho, 0)
    else:  # one tile (profiling): hierarchy built without a solve, so few launches precede it
        opt.kernel.set_rho(torch.full((opt.kernel.n_elements,), CONFIGS[cfg_name]["vf"] ** 3, dtype=torch.float64,
                                      device="cuda"))
        opt.solver._configure()
        _lib.call("edge_mg_setup", h)
    torch.cuda.synchronize()
    prec = 1 if args.precision == "mixed" else 0
    nvar = 5 if args.precision == "fp64" else (16 if _lib.lib().edge_uses_cube_form(h) else 9)
    k = opt.kernel
    n_dof, n_el = k.shape[0], k.n_elements
    w = 8 if args.precision == "fp64" else 4
    plain_bytes = 2 * w * n_dof + w * n_el
    sweep_bytes = plain_bytes + n_dof * (w + (8 if args.precision == "fp64" else 2) + 0)
    peak, kind = peaks()
    rows = []
    ms = ctypes.c_double()
    variants = [args.tile] if args.tile is not None else list(range(nvar))
    bps_list = [args.tile_bps] if args.tile is not None else [2, 4, 8, 16]
    for v in variants:
        for bps in bps_list:
            r = {"variant": v, "bps": bps}
            for sweep in (0, 1):
                _lib.call("edge_time_fine", h, prec, v, bps, sweep, max(1, args.steps), ctypes.byref(ms))
                b = sweep_bytes if sweep else plain_bytes
                r["sweep_us" if sweep else "plain_us"] = round(ms.value * 1e3, 2)
                r["sweep_frac" if sweep else "plain_frac"] = round(b / (ms.value / 1e3) / 1e9 / peak, 3)
            rows.append(r)
    levels = []
    cfg = CONFIGS[cfg_name]
    for lvl in range(1, cfg["n_level"]):
        ne = [v >> lvl for v in cfg["nel"]]
        nodes = (ne[0] + 1) * (ne[1] + 1) * (ne[2] + 1)
        # stencil (123 coefficients; BF16 copies in mixed precision) + u, b, Dinv, out per node
        b = nodes * (123 * (2 if args.precision == "mixed" else w) + 4 * 3 * w)
        row = {"level": lvl, "nodes": nodes}
        for name, qmax, pair, tiled in (("thread", 0, -1, -1), ("pair", 0, 0, -1), ("quad", 1 << 40, -1, -1),
                                        ("tiled", 0, 0, 0)):
            _lib.call("edge_set_stencil_quad", h, qmax)
            _lib.call("edge_set_stencil_pair", h, pair)
            _lib.call("edge_set_stencil_tiled", h, tiled)
            if tiled >= 0:
                _lib.call("edge_mg_setup", h)  # fills the tile-major copies
            _lib.call("edge_time_level", h, lvl, max(1, args.steps), ctypes.byref(ms))
            row[name + "_us"] = round(ms.value * 1e3, 2)
            row[name + "_frac"] = round(b / (ms.value / 1e3) / 1e9 / peak, 3)
        _lib.call("edge_set_stencil_pair", h, 200000)
        _lib.call("edge_set_stencil_tiled", h, 200000)
        levels.append(row)
    _lib.call("edge_set_stencil_quad", h, 40000)
    return {"mode": "tiles", "workload": cfg_name, "precision": args.precision, "peak_GBps": peak,
            "peak_source": kind, "plain_bytes": plain_bytes, "sweep_bytes": sweep_bytes, "tiles": rows,
            "stencil_levels": levels}


def run_analysis(args, cfg_name):
    """Profiling helper: one SIMP analysis (filter, SIMP law, solve, sensitivities) of the
    workload at rho = vf with the fine tile, the per-level sweeps, the persistent-tail level
    and maxiter pinned (--tile/--tile-bps, --sweeps, --tail, --maxiter) and no autotuning, so a
    profiler sees a fixed, short sequence of launches (--no-graph: every kernel its own launch).
    Prints its own JSON line."""
    import torch
    from edge_to_b200 import _lib
    cfg = CONFIGS[cfg_name]
    opt, rho = build_problem(cfg, args.precision, args.n_smooth, graph=not args.no_graph)
    sv = opt.solver
    sv.autotune = False
    sv.tune_sweeps = False
    if args.fixed_omega and args.precision == "mixed":
        sv.mixed_omega = "max"
        sv._omega_mode = "fixed"
    sv._configure()
    h = opt.kernel.handle
    _lib.call("edge_set_fine_tile", h, 10 if args.tile is None else args.tile, args.tile_bps)
    if args.fuse_xr:
        _lib.call("edge_set_fuse_xr", h, 1)
    if args.sweeps:
        pat = [int(v) for v in args.sweeps.split(",")]
        _lib.call("edge_mg_set_sweeps", h, _lib.int_array(pat), len(pat))
    _lib.call("edge_set_tail", h, args.tail)
    if args.no_fuse:
        _lib.call("edge_set_fuse", h, 0)
    sv.maxiter = args.maxiter
    c, dr, res = opt.solve_and_process(rho, 0)
    torch.cuda.synchronize()
    return {"mode": "analysis", "workload": cfg_name, "precision": args.precision, "pcg_iters":
            opt.last_stats.get("pcg_iters"), "residual": res, "compliance": float(c)}


def run_batch(args):
    """Batching configuration: randomized 2-D problems of uneven size (edge_to_b200.batch);
    by default every SIMP stage's solves and OC updates run as one persistent launch each
    (BatchSIMP(persistent=True)), else per-problem solve graphs on host threads with one CUDA
    stream each; value = problem-iterations per second (one SIMP iteration of one problem =
    filter + SIMP law + GMG-PCG solve + sensitivities + OC).
    With N ranks every rank solves its own batch_size problems (batch.shard_specs: disjoint
    seeded problems, no collective on the data path; weak scaling), timed between barriers
    and taken over the slowest rank."""
    import numpy as np
    import torch
    from edge_to_b200 import batch
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    n = args.batch_size
    specs = batch.shard_specs(n, rank, seed=0)
    persistent = args.batch_mode == "persistent"
    sweeps = tuple(int(v) for v in args.batch_sweeps.split(",")) if (persistent and args.batch_sweeps) else None
    max_level = args.batch_max_level if args.batch_max_level else (6 if persistent else 4)
    b = batch.BatchSIMP(specs, precision=args.precision, tol=1e-6, maxiter=1000, n_threads=args.batch_threads,
                        persistent=persistent, max_level=max_level, block_threads=args.batch_block,
                        sweeps=sweeps, team=args.batch_team, split_dof=args.batch_split)
    b.step(args.warmup)               # initial analysis, autotuners, warm-up iterations
    b.phase_ms = {}
    clocks = ClockSampler(local)
    clocks.start()
    _barrier(ws)
    ms = b.step(args.steps)
    _barrier(ws)
    clk = clocks.stop()
    ms = _max_over_ranks(ms, ws)
    pcg = [int(np.mean(it["pcg"][-args.steps:])) for it in b.items]
    dofs = [2 * (sp["nelx"] + 1) * (sp["nely"] + 1) for sp in specs]
    # every rank solves its own seeded problems: their sizes and PCG work differ, so the line
    # records each rank's DOF total and DOF x PCG-iteration work beside the slowest rank's time
    work = float(sum(d * p for d, p in zip(dofs, pcg)))
    dof_per_rank = _gather_over_ranks(float(sum(dofs)), ws)
    work_per_rank = _gather_over_ranks(work, ws)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return None
    return {"metric": f"SIMP problem-iterations/s, {n} random uneven 2-D problems per GPU",
            "value": whole_job_rate(n * args.steps, ws, ms),
            "unit": "problem-iter/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32+bf16/f64",
            "data": "synthetic: seeded random problems (edge_to_b200.batch.random_spec, seed 0)",
            "config": {"workload": f"batch{n}_2d", "problems": n * ws, "problems_per_gpu": n,
                       "parallelism": f"independent problems x{ws}" if ws > 1 else "1 GPU",
                       "dof_total_rank0": int(np.sum(dofs)),
                       "dof_total_per_rank": [int(v) for v in dof_per_rank],
                       "dof_x_pcg_iters_per_step_per_rank": [int(v) for v in work_per_rank],
                       "elements_total_rank0": int(sum(sp["nelx"] * sp["nely"] for sp in specs)),
                       "rtol": 1e-6, "precision": args.precision, "mode": args.batch_mode,
                       "threads_streams": b.n_threads, "max_level": max_level,
                       "solve_launch": ({"threads_per_block": args.batch_block, "blocks_per_problem": args.batch_team,
                                         "single_block_below_dof": args.batch_split,
                                         "sweeps_fine_coarse": sweeps} if persistent else None),
                       "pcg_iters_max_rank0": int(max(max(it["pcg"][-args.steps:]) for it in b.items)),
                       "phase_ms_per_step_rank0": ({k: v / args.steps for k, v in b.phase_ms.items()}
                                                   if persistent else None),
                       "padded_problems_rank0": int(sum(it["opt"].solver.padded for it in b.items)),
                       "pcg_iters_mean_rank0": float(np.mean(pcg))},
            "clocks": clk}


def run_reference(args, cfg_name):
    """The reference's CPU path on this host's cores (oracle/cpu_simp.py), rank 0 only."""
    ws, rank, local = dist_env()
    if rank != 0:
        return None
    cores = os.cpu_count() or 1
    m = finish_cpu_reference(start_cpu_reference(cfg_name, min(max(1, args.steps), CPU_PCG_SAMPLES), cores), 1800.0)
    cb = cpu_reference_line(m)
    v = cb["value"]
    t = m.get("seconds_per_iteration")
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3 if t else None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": cfg_name, "precision": "fp64", "parallelism": f"host cores ({cores})",
                       "pcg_samples": len(m.get("pcg_iteration_samples_s", []))},
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="skip timing the plain FP64 path beside the mixed-precision one")
    ap.add_argument("--config", default="cantilever_256x128x128", choices=list(CONFIGS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-oracle-trajectory", action="store_true",
                    help="skip the FP64 trajectory at rtol 1e-10 the timed paths are compared with")
    ap.add_argument("--no-fuse", action="store_true",
                    help="mixed path: the fine level's sweeps and search direction as separate launches")
    ap.add_argument("--no-kind-tune", action="store_true",
                    help="mixed path: one fine tile for the three fused launch kinds (default: the autotuner may "
                         "give each kind its own)")
    ap.add_argument("--galerkin", default="axis", choices=["axis", "direct"],
                    help="3-D Galerkin products of levels >= 2: three one-axis passes (default) or one direct pass")
    ap.add_argument("--stencil", default="default", choices=["default", "linear", "tiled"],
                    help="mixed path, coarse levels of 200k slots and more: linear BF16 stencil copy (k_st3_apply2) "
                         "or tile-major copy (k_st3_apply2t)")
    ap.add_argument("--fuse-xr", action="store_true",
                    help="mixed path: the PCG's x/r update folded into the next iteration's fine launches when "
                         "the smoother weight is fixed (default: its own launch, faster at 12.8M DOF)")
    ap.add_argument("--fixed-omega", action="store_true",
                    help="analysis mode: the mixed path's smoother weight fixed at omega (the autotuner's other choice)")
    ap.add_argument("--omega-schedule", action="store_true",
                    help="mixed path: the reference's residual-driven smoother weight (default: fixed at omega)")
    ap.add_argument("--mode", default="simp", choices=["simp", "matvec", "tiles", "analysis"])
    ap.add_argument("--maxiter", type=int, default=12, help="analysis mode: PCG iteration limit")
    ap.add_argument("--tail", type=int, default=0,
                    help="analysis mode: level from which the V-cycle is one persistent launch (0 = off)")
    ap.add_argument("--tile", type=int, default=None, help="matvec/tiles mode: fine-kernel tile variant (0-15)")
    ap.add_argument("--tile-bps", type=int, default=8, help="matvec mode: y-chunking target (blocks per SM)")
    ap.add_argument("--n-smooth", type=int, default=3,
                    help="default smoothing sweeps of the timed path (the FP64 path keeps the reference's 3)")
    ap.add_argument("--coarse-fp32", action="store_true",
                    help="mixed path: apply the coarse stencils in FP32 (default: BF16 copies)")
    ap.add_argument("--residual64", action="store_true", help="mixed path: FP64-stored residual recurrence")
    ap.add_argument("--pdl", action="store_true",
                    help="solve graph with programmatic dependent launch (default: plain stream order)")
    ap.add_argument("--sweeps", default=None,
                    help="per-level smoothing sweeps of the timed path, e.g. 1,1,1,1,1 (no sweep autotuning)")
    ap.add_argument("--no-graph", action="store_true",
                    help="host-driven PCG loop instead of one CUDA graph per solve (same launches; for profilers)")
    ap.add_argument("--batch", action="store_true",
                    help="the batching configuration (random uneven 2-D problems) instead of --config")
    ap.add_argument("--batch-size", type=int, default=256)
    ap.add_argument("--batch-threads", type=int, default=16, help="batch, threads mode: host threads / streams")
    ap.add_argument("--batch-mode", default="persistent", choices=["threads", "persistent"],
                    help="batch: every solve and OC update of a SIMP stage in one persistent launch (default), or "
                         "per-problem solve graphs on host threads")
    ap.add_argument("--batch-max-level", type=int, default=0,
                    help="batch: deepest multigrid per problem (0: 6 persistent, 4 threads)")
    ap.add_argument("--batch-block", type=int, default=1024, choices=[256, 512, 1024],
                    help="batch, persistent mode: threads per block of the solve launch")
    ap.add_argument("--batch-team", type=int, default=4, choices=[1, 2, 4, 8],
                    help="batch, persistent mode: blocks (a thread block cluster) per problem")
    ap.add_argument("--batch-split", type=int, default=0,
                    help="batch, persistent mode: problems below this many DOFs solved by single blocks beside the teams")
    ap.add_argument("--batch-sweeps", default="1,2",
                    help="batch, persistent mode: smoothing sweeps on the fine level and on coarser levels")
    ap.add_argument("--breakdown", action="store_true",
                    help="extra untimed step with per-category launch timing (events on every launch)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.impl == "reference":
        line = run_reference(args, args.config)
    elif args.batch:
        line = run_batch(args)
    elif args.mode == "matvec":
        line = run_matvec(args, args.config)
    elif args.mode == "tiles":
        line = run_tiles(args, args.config)
    elif args.mode == "analysis":
        line = run_analysis(args, args.config)
    else:
        line = run_ours(args, args.config)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
