#!/usr/bin/env python
"""Benchmark of the SIMP analysis-and-sensitivity step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    (N > 1: launched by torch.distributed.run, one rank per GPU)

Default line (--workload headline): the 384x128x128 Hex8 half-MBB beam
(19,220,355 DOF), seeded smooth density field; one step = SIMP moduli, the
mixed-precision GMG-PCG solve to ||r||/||f|| <= 1e-8 (FP32 V-cycle, FP64
residual), compliance and sensitivities; value = numeq x the Jacobi-PCG
iterations this system needs to 1e-8 / step time (the reference algorithm's
DOF*iter, so the ratio to the reference arm is the time-to-solution
speed-up); the reference arm times the oracle's matrix-free Jacobi-PCG on the
same system on the host cores.  See headline_ours for the extra keys.

--workload c2 (one step): the 192x64x64 Hex8 cantilever (2,446,275 DOF, numeq
2,433,600): x = 0 face clamped, unit line load in -z along the bottom edge of
the x = L face, E0 = 1, Emin = 1e-9, nu = 0.3, p = 3, densities i.i.d.
U[0.01, 1] from a seed; solve K(rho) u = f to ||r||/||f|| <= 1e-8, then
compliance and element sensitivities.  Synthetic inputs; every rank solves
its own seeded instance (replicas, weak scaling).

Metric: PCG DOF*iter/s = numeq x (operator applications in the Krylov loop)
/ step time, with the ICARAT Eigen_CG algorithm (Jacobi-preconditioned CG in
FP64) on both arms, so the ratio of the two arms is the time-to-solution
speed-up.  `value` is device-resident (density already in HBM); `e2e` goes
through the C ABI with pinned host buffers (density in; displacement,
compliance and sensitivities out) inside the timed region.

--impl reference times the oracle's CPU restatement of ICARAT's path
(assembled CSR + Eigen-semantics Jacobi-PCG, all host threads) on a bounded
sample of PCG iterations of the same problem.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "icarat-contact_b200", "python"), os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

WORKLOAD = ("cantilever3d", (192, 64, 64))
TOL = 1e-8
SEED = 2024
METRIC = "PCG DOF*iter/s (FP64 Jacobi-PCG, Eigen_CG semantics), 1e-8"
UNIT = "DOF*iter/s"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            P = json.load(f)
        return float(P["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic(kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


# ----------------------------------------------------------------- clocks --
_CLK_FIELDS = ["index", "clocks.sm", "clocks.max.sm", "power.draw",
               "clocks_event_reasons.active", "clocks_event_reasons.hw_slowdown",
               "clocks_event_reasons.hw_thermal_slowdown",
               "clocks_event_reasons.sw_thermal_slowdown", "clocks_event_reasons.sw_power_cap"]


def clocks_start(gpu):
    try:
        return subprocess.Popen(
            ["nvidia-smi", "--query-gpu=" + ",".join(_CLK_FIELDS), "--format=csv,noheader,nounits",
             "-lms", "200", "-i", str(gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
            text=True)
    except Exception:
        return None


def clocks_stop(proc):
    if proc is None:
        return None
    time.sleep(0.25)
    proc.terminate()
    try:
        out, _ = proc.communicate(timeout=5)
    except Exception:
        proc.kill()
        out = ""
    sm, mx, reasons = [], [], set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for line in out.strip().splitlines():
        f = [x.strip() for x in line.split(",")]
        if len(f) < 9:
            continue
        try:
            sm.append(float(f[1]))
            mx.append(float(f[2]))
        except ValueError:
            continue
        for k, v in zip(names, f[5:9]):
            if v.lower().startswith("active"):
                reasons.add(k)
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
            "samples": len(sm)}


# -------------------------------------------------------------- reference --
def run_cpu_sample(nit, reps=1):
    """Oracle (assembled CSR + Jacobi-PCG) on the bench problem: seconds per
    `nit` PCG iterations, numeq, threads, assembly seconds."""
    import ctypes as C

    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import pyoracle as po
    kind, n = WORKLOAD
    p = cases.build_oracle(kind, *n)
    rho = cases.uniform_density(p.nel, SEED)
    dof, numeq = p.dofs()
    f = p.fext()
    t0 = time.perf_counter()
    h = po.lib().orc_csr_assemble(C.byref(p.g), dof.ctypes.data_as(C.POINTER(C.c_int)), numeq,
                                  rho.ctypes.data_as(C.POINTER(C.c_double)))
    t_asm = time.perf_counter() - t0
    x = np.zeros(numeq)
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        po.lib().orc_csr_pcg_fixed(h, f.ctypes.data_as(C.POINTER(C.c_double)),
                                   x.ctypes.data_as(C.POINTER(C.c_double)), nit)
        times.append(time.perf_counter() - t0)
    po.lib().orc_csr_free(h)
    return times, numeq, po.lib().orc_num_threads(), t_asm


def reduce_over_ranks(ms, units, dist, device):
    """Whole-job figures of a replica run: the slowest rank's time and the
    units every rank processed (max and sum over ranks)."""
    if dist is None:
        return ms, units
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    u = torch.tensor([units], dtype=torch.float64, device=device)
    dist.all_reduce(u)
    return float(t.item()), float(u.item())


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    nit = 10
    times, numeq, threads, t_asm = run_cpu_sample(nit, reps=args.warmup + args.steps)
    timed = times[args.warmup:]
    tot = sum(timed)
    value = numeq * nit * len(timed) / tot
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(timed), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded densities U[0.01,1])",
        "config": {"workload": "cantilever3d 192x64x64 Hex8", "numeq": numeq, "tol": TOL,
                   "step": f"{nit} Jacobi-PCG iterations on the assembled CSR (bounded sample)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{nit} PCG iterations per step after a {t_asm:.1f} s CSR "
                                   f"assembly of the same problem"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------- ours --
def ours_arm(args):
    import numpy as np
    import torch
    import cases
    import icarat_b200 as icb

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = icb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{local}")
    kind, n = WORKLOAD
    prob = cases.build_gpu(ctx, kind, *n)
    numeq = prob.numeq
    rho_h = cases.uniform_density(prob.nel, SEED + rank)
    rho_d = torch.from_numpy(rho_h).to(f"cuda:{local}")
    torch.cuda.synchronize()

    def step():
        prob.set_density_device(rho_d.data_ptr())
        info = prob.solve(tol=TOL, maxit=200000)
        c = prob.compliance()
        icb.lib().icb_sensitivity_device(prob.h)
        return info, c

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    barrier()
    clk = clocks_start(local) if rank == 0 else None
    l0 = icb.launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    mv, infos = 0, []
    for k in range(args.steps):
        info, comp = step()
        mv += info["matvecs"]
        infos.append(info)
        ev[k + 1].record(stream)
    e0, e1 = ev[0], ev[-1]
    barrier()
    lat = sorted(ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps))
    clocks = clocks_stop(clk)
    launches = icb.launch_count() - l0
    ms, units = reduce_over_ranks(e0.elapsed_time(e1), float(numeq) * mv, dist, f"cuda:{local}")
    value = units / (ms * 1e-3)

    # ---- e2e through the C ABI with pinned host buffers
    rho_pin = torch.from_numpy(rho_h).pin_memory()
    u_pin = torch.empty(numeq, dtype=torch.float64).pin_memory()
    dc_pin = torch.empty(prob.nel, dtype=torch.float64).pin_memory()
    import ctypes as C
    L = icb.lib()
    dptr = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))  # noqa: E731

    def step_e2e():
        icb.check(L.icb_set_density(prob.h, dptr(rho_pin)))
        info = prob.solve(tol=TOL, maxit=200000)
        c = C.c_double()
        icb.check(L.icb_compliance(prob.h, C.byref(c)))
        icb.check(L.icb_sensitivity(prob.h, dptr(dc_pin), None))
        icb.check(L.icb_get_displacement(prob.h, dptr(u_pin)))
        return info

    step_e2e()
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    mv2 = 0
    for _ in range(args.steps):
        mv2 += step_e2e()["matvecs"]
    f1.record(stream)
    barrier()
    ms2, units2 = reduce_over_ranks(f0.elapsed_time(f1), float(numeq) * mv2, dist, f"cuda:{local}")
    e2e = {"value": units2 / (ms2 * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": 8 * prob.nel,
           "d2h_bytes_per_step": 8 * (numeq + prob.nel + 1)}

    # ---- roofline of the dominant kernel (FP64 operator), timed live with
    # an L2 flush before every launch
    prob.set_density_device(rho_d.data_ptr())
    t_mv = op_launch_seconds(prob, icb.FP64, stream, local)
    ndof = prob.neq
    alg_bytes = 8 * (2 * ndof + prob.nel)
    flops = 207 * prob.nel
    peak, peak_kind = _peaks()
    achieved = alg_bytes / t_mv / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": _traffic("matvec_h8m_fp64_cantilever3d_192x64x64"),
                "kernel": "k_matvec_h8m<double>", "launch_us": t_mv * 1e6,
                "peak_source": peak_kind,
                "fp64_tflops": flops / t_mv / 1e12,
                "note": "FP64 corner-mode element operator: 207 flop per element "
                        "(two butterflies + 45 multiply-adds; the dense 24x24 form is 1152)"}

    # ---- the same solve with the multigrid paths (time to solution)
    alt = {}
    for name, kw in (("fp64_gmg", dict(precision=icb.FP64, precond=icb.GMG)),
                     ("mixed_gmg", dict(precision=icb.MIXED, precond=icb.GMG))):
        prob.set_density_device(rho_d.data_ptr())
        prob.solve(tol=TOL, maxit=20000, raise_on_error=False, **kw)  # builds the hierarchy
        h0, h1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        h0.record(stream)
        inf = prob.solve(tol=TOL, maxit=20000, raise_on_error=False, **kw)
        h1.record(stream)
        torch.cuda.synchronize()
        t = h0.elapsed_time(h1)
        alt[name] = {"ms": t, "iters": inf["iters"], "true_relres": inf["true_relres"],
                     "status": icb.STATUS.get(inf["rc"], inf["rc"]),
                     "speedup_vs_fp64_jacobi": (ms / args.steps) / t if inf["rc"] == 0 else None}

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded densities U[0.01,1], one instance per rank)",
            "config": {"workload": "cantilever3d 192x64x64 Hex8 (2,446,275 DOF)", "numeq": numeq,
                       "tol": TOL, "parallelism": f"replicas x{world}",
                       "l2": "working set ~150 MB per rank > 126 MB L2 (no flush)"},
            "solve": {"iters": infos[-1]["iters"], "matvecs": infos[-1]["matvecs"],
                      "relres": infos[-1]["relres"], "true_relres": infos[-1]["true_relres"],
                      "compliance": comp},
            "latency_ms": {"p50": lat[len(lat) // 2], "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "time_to_solution": alt,
            "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu:
        nit = 10
        times, ne, threads, t_asm = run_cpu_sample(nit, reps=2)
        cv = ne * nit / min(times)
        line["cpu_baseline"] = {"value": cv, "unit": UNIT, "cores": threads, "kind": "port",
                                "sample": f"{nit} Jacobi-PCG iterations on the assembled CSR of "
                                          f"the same problem (assembly {t_asm:.1f} s, untimed)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    prob.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------ headline (c3) --
C3_GRID = (384, 128, 128)
C3_METRIC = ("PCG DOF*iter/s at 1e-8, Eigen_CG-equivalent: numeq x the Jacobi-PCG iterations "
             "this system needs to ||r||/||f|| <= 1e-8, per second of analysis-and-sensitivity "
             "step (mixed-precision GMG-PCG on ours, Jacobi-PCG on the reference)")


def c3_config(grid):
    nx, ny, nz = grid
    dof = 3 * (nx + 1) * (ny + 1) * (nz + 1)
    return {"workload": f"halfmbb3d {nx}x{ny}x{nz} Hex8 ({dof:,} DOF), seeded smooth density "
                        f"field on [0.001,1], E0=1, Emin=1e-9, nu=0.3, p=3, tol 1e-8",
            "tol": TOL,
            "l2": "inputs larger than L2: one FP64 field vector is 154 MB > 126 MB"}


def c3_cpu_sample(grid, nit, seed):
    """The oracle's matrix-free Jacobi-PCG (the Eigen_CG algorithm; the assembled
    matrix of this grid needs ~77 GB) on the host cores: seconds per `nit`
    iterations, numeq, threads."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import cases
    import pyoracle as po
    o = cases.build_oracle("halfmbb3d", *grid)
    rho = smooth_field(*grid, seed=seed)
    _, numeq = o.dofs()
    return (lambda: o.ebe_pcg_time(rho, nit)[0]), numeq, po.lib().orc_num_threads()


def headline_reference(args):
    """--impl reference: the CPU restatement of ICARAT's Eigen_CG solve on the
    same c3 problem, each step a bounded sample of `nit` Jacobi-PCG iterations;
    rank 0 only."""
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    grid = tuple(args.size) if args.size else C3_GRID
    nit = 10
    run, numeq, threads = c3_cpu_sample(grid, nit, SEED)
    for _ in range(args.warmup):
        run()
    times = [run() for _ in range(args.steps)]
    tot = sum(times)
    value = numeq * nit * len(times) / tot
    sample = (f"{nit} matrix-free Jacobi-PCG iterations per step (Eigen_CG semantics, the "
              f"oracle's restatement; {tot / len(times) / nit:.3f} s per iteration on {threads} "
              f"threads)")
    print(json.dumps({
        "impl": "reference", "metric": C3_METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * tot / len(times), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded smooth density field)",
        "config": c3_config(grid),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
        flush=True)
    return 0


def headline_ours(args):
    """The default bench line: c3, the 384x128x128 Hex8 half-MBB beam.  One step
    is the analysis-and-sensitivity step on device-resident densities: SIMP
    moduli, the mixed-precision GMG-PCG solve to ||r||/||f|| <= 1e-8 (FP64
    residual), compliance and element sensitivities.  The value counts the
    work of the reference algorithm (numeq x its Jacobi-PCG iteration count
    to 1e-8, measured on the same system) per second of step, so the ratio to
    the reference arm is the time-to-solution speed-up; the raw GMG-PCG
    DOF*iter/s, the FP64 GMG and FP64 Jacobi solves of the same system and the
    errors of the mixed solve against the FP64 one are reported beside it."""
    import ctypes as C

    import numpy as np
    import torch
    import cases
    import icarat_b200 as icb

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    grid = tuple(args.size) if args.size else C3_GRID
    ctx = icb.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=dev)
    prob = cases.build_gpu(ctx, "halfmbb3d", *grid)
    numeq = prob.numeq
    rho_h = smooth_field(*grid, seed=SEED + rank)
    rho_d = torch.from_numpy(rho_h).to(dev)
    torch.cuda.synchronize()

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def timed(fn):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        r = fn()
        b.record(stream)
        torch.cuda.synchronize()
        return r, a.elapsed_time(b)

    # the reference algorithm on this system: FP64 Jacobi-PCG (Eigen_CG) to 1e-8
    prob.set_density_device(rho_d.data_ptr())
    inf_j, ms_j = timed(lambda: prob.solve(precision=icb.FP64, precond=icb.JACOBI, tol=TOL,
                                           maxit=200000))
    n_jacobi = inf_j["iters"]
    comp_j = prob.compliance()
    # the plain FP64 GPU path with the same preconditioner: FP64 GMG-PCG
    prob.solve(precision=icb.FP64, precond=icb.GMG, tol=TOL, maxit=20000)  # builds the hierarchy
    inf_g, ms_g = timed(lambda: prob.solve(precision=icb.FP64, precond=icb.GMG, tol=TOL,
                                           maxit=20000))
    comp_g = prob.compliance()
    dc_g = prob.sensitivity()

    mixed = dict(precision=icb.MIXED, precond=icb.GMG, tol=TOL, maxit=20000)

    def step():
        prob.set_density_device(rho_d.data_ptr())
        info = prob.solve(**mixed)
        c = prob.compliance()
        icb.lib().icb_sensitivity_device(prob.h)
        return info, c

    for _ in range(args.warmup):
        step()
    barrier()
    clk = clocks_start(local) if rank == 0 else None
    l0 = icb.launch_count()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    ev[0].record(stream)
    infos = []
    for k in range(args.steps):
        info, comp = step()
        infos.append(info)
        ev[k + 1].record(stream)
    barrier()
    clocks = clocks_stop(clk)
    launches = icb.launch_count() - l0
    lat = sorted(ev[k].elapsed_time(ev[k + 1]) for k in range(args.steps))
    ms, units = reduce_over_ranks(ev[0].elapsed_time(ev[-1]), float(numeq) * n_jacobi * args.steps,
                                  dist, dev)
    _, raw_units = reduce_over_ranks(0.0, float(numeq) * sum(i["iters"] for i in infos), dist, dev)
    value = units / (ms * 1e-3)
    comp_m = prob.compliance()
    dc_m = prob.sensitivity()
    err = {"compliance_rel_vs_fp64_gmg": abs(comp_m - comp_g) / abs(comp_g),
           "sens_linf_rel_vs_fp64_gmg": float(np.abs(dc_m - dc_g).max() / np.abs(dc_g).max()),
           "compliance_rel_vs_fp64_jacobi": abs(comp_m - comp_j) / abs(comp_j)}

    # ---- e2e: the C ABI with pinned host buffers (density in; compliance,
    # sensitivities and displacement out) inside the timed region
    rho_pin = torch.from_numpy(rho_h).pin_memory()
    u_pin = torch.empty(numeq, dtype=torch.float64).pin_memory()
    dc_pin = torch.empty(prob.nel, dtype=torch.float64).pin_memory()
    L = icb.lib()
    dptr = lambda t: C.cast(C.c_void_p(t.data_ptr()), C.POINTER(C.c_double))  # noqa: E731

    def step_e2e():
        icb.check(L.icb_set_density(prob.h, dptr(rho_pin)))
        prob.solve(**mixed)
        c = C.c_double()
        icb.check(L.icb_compliance(prob.h, C.byref(c)))
        icb.check(L.icb_sensitivity(prob.h, dptr(dc_pin), None))
        icb.check(L.icb_get_displacement(prob.h, dptr(u_pin)))

    step_e2e()
    barrier()
    _, ms2 = timed(lambda: [step_e2e() for _ in range(args.steps)])
    ms2, units2 = reduce_over_ranks(ms2, float(numeq) * n_jacobi * args.steps, dist, dev)
    e2e = {"value": units2 / (ms2 * 1e-3), "unit": UNIT, "ms_per_step": ms2 / args.steps,
           "h2d_bytes_per_step": 8 * prob.nel, "d2h_bytes_per_step": 8 * (numeq + prob.nel + 1)}

    # ---- roofline: the dominant kernel of the step is the V-cycle's FP32
    # Chebyshev smoother on the fine level (the element operator with its fused
    # update: 37 % of the solve's device time in the launch list); beside it the
    # same FP32 operator without the update and the FP64 operator of the outer
    # iteration.  Each timed live with an L2 flush before every launch.
    prob.set_density_device(rho_d.data_ptr())
    peak, peak_kind = _peaks()
    rows = {}
    k32 = "k_matvec_h8p<float>" if icb.get_option("hex8_pair") == 1 else "k_matvec_h8m<float>"
    vec = 3 * prob.nnode  # entries of one field vector the kernels touch
    for name, prec, es, kern, cheb in (
            ("fp32_cheb", icb.MIXED, 4, k32 + " OP_CHEB", True),
            ("fp32_apply", icb.MIXED, 4, k32, False),
            ("fp64", icb.FP64, 8, "k_matvec_h8m<double>", False)):
        # u, b, D^-1 and the previous iterate read, y written, the moduli and
        # the constraint flags; the plain operator reads u and writes y.  All
        # three move more than the 126 MB L2 per launch: timed back to back
        b = es * ((5 if cheb else 2) * vec + prob.nel) + (prob.nnode if cheb else 0)
        t = op_launch_seconds(prob, prec, stream, local, cheb=cheb, flush_l2=False)
        tkey = (k32 + ("_cheb" if cheb else "")) if prec == icb.MIXED else kern
        rows[name] = {"bound": "hbm", "achieved": b / t / 1e9, "peak": peak, "unit": "GB/s",
                      "frac": b / t / 1e9 / peak, "kernel": kern, "launch_us": t * 1e6,
                      "alg_bytes": b, "peak_source": peak_kind,
                      "l2": "inputs larger than L2, launches back to back",
                      "traffic": _traffic(f"{tkey}_384x128x128")}
    roofline = dict(rows["fp32_cheb"])
    roofline["fp32_operator_alone"] = rows["fp32_apply"]
    roofline["fp64_outer_operator"] = rows["fp64"]

    # ---- the topology-optimisation loop on the same beam: 20 MMA steps with
    # the Helmholtz filter (R = 3, volume fraction 0.3), mixed solves
    topo = None
    if args.mma_steps > 0:
        steps = args.mma_steps
        o = icb.loop_opts(steps, 3.0, precision=icb.MIXED, volume_ref=0.3 * float(np.prod(grid)))
        its = np.zeros(steps)
        o.iter_seconds = its.ctypes.data_as(icb._dp)
        hist, x = np.zeros(steps), np.zeros(prob.nel)
        t0 = time.perf_counter()
        icb.check(L.icb_run_mma(prob.h, C.byref(o), icb._p(rho_h), icb._p(hist), icb._p(x)))
        dt = time.perf_counter() - t0
        topo = {"iter_per_s": steps / dt, "steps": steps,
                "step_ms_p50": 1e3 * float(np.median(its)),
                "step_ms_p99": 1e3 * float(np.quantile(its, 0.99)),
                "compliance_first_last": [hist[0], hist[-1]]}

    line = {"metric": C3_METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32 multigrid / f64 Krylov and residual",
            "data": "synthetic (seeded smooth density field, one instance per rank)",
            "config": dict(c3_config(grid), parallelism=f"replicas x{world}"),
            "solve": {"iters": infos[-1]["iters"], "true_relres": infos[-1]["true_relres"],
                      "compliance": comp, "jacobi_iters_to_tol": n_jacobi,
                      "pcg_dof_iter_per_s_raw": raw_units / (ms * 1e-3)},
            "time_to_solution_ms": {"mixed_gmg_step": ms / args.steps, "fp64_gmg_solve": ms_g,
                                    "fp64_gmg_iters": inf_g["iters"], "fp64_jacobi_solve": ms_j,
                                    "fp64_jacobi_iters": n_jacobi},
            "speedups": {"mixed_step_vs_fp64_gmg_solve": ms_g / (ms / args.steps),
                         "mixed_step_vs_fp64_jacobi_solve": ms_j / (ms / args.steps)},
            "mixed_vs_fp64": err,
            "latency_ms": {"p50": lat[len(lat) // 2],
                           "p99": lat[min(len(lat) - 1, int(0.99 * len(lat)))]},
            "topopt": topo, "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches),
            "clocks": clocks}
    if rank == 0 and world == 1 and not args.no_cpu:
        nit = 10
        run, ne, threads = c3_cpu_sample(grid, nit, SEED)
        tcpu = min(run() for _ in range(2))
        line["cpu_baseline"] = {"value": ne * nit / tcpu, "unit": UNIT, "cores": threads,
                                "kind": "port",
                                "sample": f"{nit} matrix-free Jacobi-PCG iterations of the oracle "
                                          f"on the same system ({tcpu / nit:.3f} s per iteration)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    prob.close()
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()
    return 0


# ------------------------------------------------------------- workloads --
def _clock_wrap(fn):
    clk = clocks_start(int(os.environ.get("LOCAL_RANK", "0")))
    try:
        return fn(), clocks_stop(clk)
    except BaseException:
        clocks_stop(clk)
        raise


def smooth_field(nx, ny, nz, seed, lo=0.001, hi=1.0, modes=16):
    """the c3 density field (tests/cases.py holds the definition)"""
    import cases
    return cases.smooth_field(nx, ny, nz, seed, lo, hi, modes)


def op_launch_seconds(prob, prec, stream, device=0, reps=30, cheb=False, flush_l2=True):
    """Mean device time of one operator launch, each launch bracketed by CUDA
    events on the problem's stream and, with flush_l2, preceded by a write of
    256 MiB (> L2) on that stream (launches whose inputs are larger than L2 go
    back to back instead: the write-back of the flush buffer's dirty lines
    would otherwise land inside the timed launch): icb_operator_apply_device
    (y = K x), or with cheb the V-cycle's fused Chebyshev step
    icb_smoother_apply_device (c1 != 0, so it reads u, b, D^-1 and the
    previous iterate and writes y)."""
    import torch
    import icarat_b200 as icb
    dt = torch.float64 if prec == icb.FP64 else torch.float32
    nsoa = prob.soa_length()
    dev = f"cuda:{device}"
    x = torch.randn(nsoa, dtype=dt, device=dev)
    y = torch.zeros_like(x)
    b = torch.randn(nsoa, dtype=dt, device=dev)
    dinv = torch.rand(nsoa, dtype=dt, device=dev) * 0.1
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def launch():
        if cheb:
            prob.smoother_apply_device(x.data_ptr(), y.data_ptr(), b.data_ptr(), dinv.data_ptr(),
                                       0.3, 0.7, precision=prec)
        else:
            prob.operator_apply_device(x.data_ptr(), y.data_ptr(), prec)
    torch.cuda.synchronize()
    for _ in range(3):
        launch()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    with torch.cuda.stream(stream):
        for a, e in ev:
            if flush_l2:
                flush.fill_(1)
            a.record(stream)
            launch()
            e.record(stream)
    torch.cuda.synchronize()
    return sum(a.elapsed_time(e) for a, e in ev) / reps * 1e-3


def workload_operator(args):
    """The Hex8 operator y = K(rho) x in each precision and form (FP64 and
    FP32 on CUDA cores in the corner-mode and the dense form, TF32 tcgen05)
    at 192x64x64 and 384x128x128, L2 flushed before every launch;
    algorithmic bytes 8|4 x (2 x DOF + elements)."""
    import torch
    import cases
    import icarat_b200 as icb
    ctx = icb.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream())
    peak, src = _peaks()
    rows = []
    grids = [tuple(args.size)] if args.size else [(192, 64, 64), (384, 128, 128)]
    for n in grids:
        g = cases.build_gpu(ctx, "cantilever3d", *n)
        g.set_density(cases.uniform_density(g.nel, SEED))
        for name, prec, tc, modal, pair, es in (("fp64_modal", icb.FP64, 0, 1, 1, 8),
                                                ("fp64_dense", icb.FP64, 0, 0, 1, 8),
                                                ("fp32_modal_paired", icb.MIXED, 0, 1, 1, 4),
                                                ("fp32_modal_row", icb.MIXED, 0, 1, 0, 4),
                                                ("fp32_dense", icb.MIXED, 0, 0, 1, 4),
                                                ("tf32_tcgen05", icb.TF32, 1, 1, 1, 4)):
            icb.set_option("tc_operator", tc)
            icb.set_option("hex8_modal", modal)
            icb.set_option("hex8_pair", pair)
            t = op_launch_seconds(g, prec, stream)
            B = es * (2 * g.neq + g.nel)
            rows.append({"grid": "x".join(map(str, n)), "variant": name, "launch_us": t * 1e6,
                         "alg_GBps": B / t / 1e9, "frac_of_" + src: B / t / 1e9 / peak,
                         "elem_per_s": g.nel / t})
        icb.set_option("tc_operator", 0)
        icb.set_option("hex8_modal", 1)
        icb.set_option("hex8_pair", 1)
        g.close()
    print(json.dumps({"metric": "Hex8 operator launch time", "unit": "us", "rows": rows,
                      "tc_timeouts": icb.get_option("tc_timeouts"),
                      "config": {"workload": "cantilever3d densities U[0.01,1], L2 flushed"}}), flush=True)
    ctx.close()
    return 0


def workload_c1(args):
    """c1: the opt-macro-oc loop, 120x40 Q4 cantilever, cone r = 1.5, move
    0.2, threshold schedule, 50 steps; topopt iter/s on the GPU (FP64 GMG
    solves) beside the oracle's loop on the host cores."""
    import numpy as np
    import cases
    import icarat_b200 as icb
    ctx = icb.Context(0)
    g = cases.build_gpu(ctx, "cantilever2d", 120, 40)
    rho0 = np.full(g.nel, 0.5)
    icb.run_loop(g, "oc", rho0, 3, 1.5, move=0.2)
    res = {}
    for name, kw in (("fp64_jacobi", dict(precond=icb.JACOBI)), ("fp64_gmg", dict(precond=icb.GMG))):
        o = icb.loop_opts(50, 1.5, move=0.2, precond=kw["precond"])
        its = np.zeros(50)
        o.iter_seconds = its.ctypes.data_as(icb._dp)
        hist, x = np.zeros(50), np.zeros(g.nel)
        t0 = time.perf_counter()
        icb.check(icb.lib().icb_run_oc(g.h, icb.C.byref(o), icb._p(rho0), icb._p(hist), icb._p(x)))
        dt = time.perf_counter() - t0
        res[name] = {"iter_s": 50 / dt, "p50_ms": 1e3 * float(np.median(its)),
                     "p99_ms": 1e3 * float(np.quantile(its, 0.99)), "c_first": hist[0], "c_last": hist[-1]}
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    o = cases.build_oracle("cantilever2d", 120, 40)
    t0 = time.perf_counter()
    ho, xo, _ = o.oc_loop(rho0, 50, 1.5, 0.2, use_beta=True, tol=1e-8)
    dt = time.perf_counter() - t0
    best = max(v["iter_s"] for v in res.values())
    print(json.dumps({"metric": "topopt iter/s (opt-macro-oc loop, c1 120x40 Q4, 50 steps)",
                      "value": best, "unit": "iter/s", "n_gpus": 1, "higher_is_better": True,
                      "dtype": "f64", "data": "synthetic (uniform 0.5 start)",
                      "config": {"workload": "c1 cantilever2d 120x40, cone r=1.5, move 0.2, beta schedule"},
                      "paths": res,
                      "history_rel_diff_vs_oracle": float(np.max(np.abs(
                          icb.run_loop(g, "oc", rho0, 50, 1.5, move=0.2)[0] - ho) / np.abs(ho))),
                      "cpu_baseline": {"value": 50 / dt, "unit": "iter/s", "cores": po.lib().orc_num_threads(),
                                       "kind": "port", "sample": "the full 50-step loop (assembled CSR Jacobi-PCG, tol 1e-8)"}}),
          flush=True)
    return 0


def workload_c3(args):
    """c3: 384x128x128 Hex8 half-MBB (19,220,355 DOF), smooth seeded density
    field on [0.001, 1], Helmholtz R = 3, volume fraction 0.3, 20 MMA steps
    with mixed-precision GMG solves; plus the mixed solve against the FP64
    solve on the initial design."""
    import numpy as np
    import cases
    import icarat_b200 as icb
    n = tuple(args.size) if args.size else (384, 128, 128)
    steps = args.mma_steps
    ctx = icb.Context(0)
    g = cases.build_gpu(ctx, "halfmbb3d", *n)
    rho0 = smooth_field(*n, seed=SEED)
    # mixed vs FP64 on the initial design (same densities, same tolerance)
    g.set_density(rho0)
    out = {}
    if args.loop_only:
        return _c3_loop(args, icb, g, n, steps, rho0, None, None, None, None)
    for name, prec in (("fp64_gmg", icb.FP64), ("mixed_gmg", icb.MIXED)):
        g.solve(precision=prec, precond=icb.GMG, tol=TOL, maxit=20000)
        t0 = time.perf_counter()
        inf = g.solve(precision=prec, precond=icb.GMG, tol=TOL, maxit=20000)
        dt = time.perf_counter() - t0
        out[name] = {"ms": 1e3 * dt, "iters": inf["iters"], "true_relres": inf["true_relres"],
                     "compliance": g.compliance(), "dc": g.sensitivity()}
    err = {"compliance_rel": abs(out["mixed_gmg"]["compliance"] - out["fp64_gmg"]["compliance"]) /
                             abs(out["fp64_gmg"]["compliance"]),
           "sens_linf_rel": float(np.abs(out["mixed_gmg"]["dc"] - out["fp64_gmg"]["dc"]).max() /
                                  np.abs(out["fp64_gmg"]["dc"]).max())}
    for v in out.values():
        v.pop("dc")
    # the plain FP64 GPU path (the Eigen_CG drop-in: Jacobi-PCG) on the same design
    t0 = time.perf_counter()
    inf = g.solve(precision=icb.FP64, precond=icb.JACOBI, tol=TOL, maxit=200000)
    t_j = time.perf_counter() - t0
    out["fp64_jacobi"] = {"ms": 1e3 * t_j, "iters": inf["iters"], "true_relres": inf["true_relres"],
                          "compliance": g.compliance()}
    speed = {"mixed_gmg_vs_fp64_jacobi": out["fp64_jacobi"]["ms"] / out["mixed_gmg"]["ms"],
             "mixed_gmg_vs_fp64_gmg": out["fp64_gmg"]["ms"] / out["mixed_gmg"]["ms"]}
    # host-CPU reference: the assembled matrix of this grid would need ~58 GB of
    # triplets, so the oracle's matrix-free Jacobi-PCG is timed for a few
    # iterations and scaled by the iteration count of the same FP64 Jacobi solve
    cpu = None
    if not args.no_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        o = cases.build_oracle("halfmbb3d", *n)
        nit = 3
        t_it = min(o.ebe_pcg_time(rho0, nit)[0] for _ in range(2)) / nit
        cpu_ttsol = t_it * out["fp64_jacobi"]["iters"]
        cpu = {"value": nit * o.neq / (t_it * nit), "unit": "DOF*iter/s",
               "cores": po.lib().orc_num_threads(), "kind": "port",
               "sample": f"{nit} matrix-free Jacobi-PCG iterations of the oracle on the host cores "
                         f"({t_it:.3f} s per iteration); time to the FP64 solve estimated as "
                         f"per-iteration time x {out['fp64_jacobi']['iters']} iterations = {cpu_ttsol:.0f} s"}
        speed["mixed_gmg_vs_cpu_estimate"] = cpu_ttsol / (out["mixed_gmg"]["ms"] * 1e-3)
    return _c3_loop(args, icb, g, n, steps, rho0, out, err, speed, cpu)


def _c3_loop(args, icb, g, n, steps, rho0, out, err, speed, cpu):
    """the c3 MMA + Helmholtz loop and its JSON line"""
    import numpy as np
    vol = float(np.prod(n))
    o = icb.loop_opts(steps, 3.0, precision=icb.MIXED, volume_ref=0.3 * vol)
    its = np.zeros(steps)
    o.iter_seconds = its.ctypes.data_as(icb._dp)
    hist, x = np.zeros(steps), np.zeros(g.nel)
    t0 = time.perf_counter()
    icb.check(icb.lib().icb_run_mma(g.h, icb.C.byref(o), icb._p(rho0), icb._p(hist), icb._p(x)))
    dt = time.perf_counter() - t0
    print(json.dumps({"metric": "topopt iter/s (MMA + Helmholtz loop, c3 half-MBB, mixed precision)",
                      "value": steps / dt, "unit": "iter/s", "n_gpus": 1, "higher_is_better": True,
                      "dtype": "f64 Krylov / f32 multigrid", "data": "synthetic (seeded smooth field)",
                      "config": {"workload": f"halfmbb3d {n[0]}x{n[1]}x{n[2]}", "dof": g.neq,
                                 "helmholtz_R": 3.0, "volfrac": 0.3, "steps": steps, "tol": TOL},
                      "latency_ms": {"p50": 1e3 * float(np.median(its)),
                                     "p99": 1e3 * float(np.quantile(its, 0.99))},
                      "loop_seconds": dt, "step_seconds_sum": float(its.sum()),
                      "solve_initial_design": out, "mixed_vs_fp64": err, "speedups": speed,
                      "cpu_baseline": cpu, "compliance_history": hist.tolist()}), flush=True)
    return 0


def workload_batched(args):
    """c4: seeded 2D instances (nelx log-uniform 64-1024, aspect U[1,4], vf
    U[0.2,0.6], r U[1.2,4], one clamped edge, 1-4 unit point loads), OC loop
    with mixed-precision GMG solves, through icb_run_batch three ways: one
    run at a time (the sequential baseline), one stream per instance with
    host workers, and fused (every loop advancing together, the solves of all
    instances as one batched launch per kernel).  Instance-iterations/s of
    each, results checked bitwise against the sequential runs."""
    import numpy as np
    import cases
    import icarat_b200 as icb
    N = args.instances
    icb.set_option("batch_handoff", args.handoff)
    rng = np.random.default_rng(4)
    insts = [cases.random_instance2d(rng) for _ in range(N)]
    # several GPUs: every rank runs its footprint-balanced share, no exchange
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        fp = [icb.job_footprint(cases.grid_desc(i), icb.JOB_OC) for i in insts]
        insts = [insts[k] for k in icb.shard_by_footprint(fp, world)[rank]]
    Nloc = len(insts)
    nel_total = sum(i["nx"] * i["ny"] for i in insts)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    ctxs = [icb.Context(dev) for _ in range(Nloc)]
    probs = [cases.build_instance(c, i) for c, i in zip(ctxs, insts)]
    rho0 = [np.full(p.nel, i["vf"]) for p, i in zip(probs, insts)]

    def run(steps, fused, workers):
        icb.set_option("batch_fused", int(fused))
        opts = [icb.loop_opts(steps, i["r"], move=0.2, precision=icb.MIXED) for i in insts]
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        H, X, S = icb.run_batch(probs, [icb.JOB_OC] * Nloc, opts, rho0, nworkers=workers)
        dt = time.perf_counter() - t0
        if dist is not None:
            import torch
            t = torch.tensor([dt], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        icb.set_option("batch_fused", 1)
        return {"seconds": dt, "inst_iter_s": N * steps / dt, "all_ok": bool((S == 0).all()),
                "steps": steps}, H, X

    short = args.loop_steps_short
    # hierarchies, filters and graphs built once for both paths (not timed)
    run(2, True, 1)
    run(2, False, 1)
    seq, Hs, Xs = run(short, False, 1)
    runs = {"sequential": seq}
    same = True
    if "streams" in args.batch_modes:
        streams, Hw, Xw = run(short, False, args.workers[-1])
        runs[f"streams_{args.workers[-1]}_workers"] = streams
        same = same and all(np.array_equal(a, b) for a, b in zip(Hs + Xs, Hw + Xw))
    fused_short, Hf, Xf = run(short, True, 1)
    fused_short["phase_s"] = [icb.get_option(f"fused_phase_us_{k}") * 1e-6 for k in range(5)]
    fused_short["iterations_batch_vs_problems"] = [icb.get_option("fused_batch_iters"),
                                                   icb.get_option("fused_problem_iters")]
    # the batched solves' graph launches by the share of designs still
    # iterating: > 1/2, > 1/8, <= 1/8 (seconds, launches)
    fused_short["solve_by_active_share"] = {
        "s": [icb.get_option(f"fused_active_us_{k}") * 1e-6 for k in range(3)],
        "launches": [icb.get_option(f"fused_active_launches_{k}") for k in range(3)]}
    same = same and all(np.array_equal(a, b) for a, b in zip(Hs + Xs, Hf + Xf))
    runs["fused_short"] = fused_short
    fused, _, _ = run(args.loop_steps, True, 1)
    fused["phase_s"] = [icb.get_option(f"fused_phase_us_{k}") * 1e-6 for k in range(5)]
    runs["fused"] = fused
    for p in probs:
        p.close()
    for c in ctxs:
        c.close()
    if dist is not None:
        dist.destroy_process_group()
        if rank != 0:
            return 0
    print(json.dumps({"metric": "instance-iterations/s (c4 batched 2D OC)", "value": fused["inst_iter_s"],
                      "unit": "instance-iter/s", "n_gpus": world, "higher_is_better": True,
                      "scaling": "strong (the instances are split over the GPUs by footprint)",
                      "dtype": "f64 Krylov / f32 multigrid", "data": "synthetic (seeded instances)",
                      "config": {"workload": f"{N} 2D Q4 instances, {nel_total} elements on rank 0",
                                 "oc_steps": args.loop_steps,
                                 "oc_steps_vs_sequential": args.loop_steps_short,
                                 "handoff": icb.get_option("batch_handoff")},
                      "speedup_vs_sequential": fused_short["inst_iter_s"] / seq["inst_iter_s"],
                      "bitwise_equal_to_sequential": same,
                      "fused_phases": "build, per-instance set-up launches, batched multigrid "
                                      "set-up and solve, compliance/sensitivity/filters, OC and wait",
                      "runs": runs}), flush=True)
    return 0


def workload_serving(args):
    """c5: Poisson job arrivals at each rate lambda into one icb_server (HBM
    budget 150 GB).  Jobs: 70 % 2D Q4 OC (nelx U[64,1024], aspect 2:1), 30 %
    3D Hex8 MMA (nelx U[32,128], nely = nelz = nelx/2), vf U[0.2,0.5],
    r U[1.5,3]; steps U[50,200] scaled by --iter-scale.  The same seeded job
    set is submitted at every rate (only the arrival gaps differ), so jobs/s
    compares one workload across loads.  Per rate: jobs/s (completed /
    makespan), p50/p99 job latency (submit to end) and iteration latency;
    finally one job re-run alone against its mixed run."""
    import numpy as np
    import cases
    import icarat_b200 as icb
    rates = args.rates
    out = {}
    probe = None
    rng = np.random.default_rng(5000)
    jobs, first, same_all = [], {}, True
    for _ in range(args.jobs_per_rate):
        if rng.uniform() < 0.7:
            inst = cases.random_instance2d(rng, nelx_range=(64, 1024), aspect_fixed=2.0,
                                           vf_range=(0.2, 0.5), r_range=(1.5, 3.0))
            kind = icb.JOB_OC
        else:
            inst = cases.random_instance3d(rng, nelx_range=(32, 128), vf_range=(0.2, 0.5),
                                           r_range=(1.5, 3.0))
            kind = icb.JOB_MMA
        nsteps = max(1, int(round(rng.integers(50, 201) * args.iter_scale)))
        nel = inst["nx"] * inst["ny"] * (inst["nz"] if inst["dim"] == 3 else 1)
        loop = icb.loop_opts(nsteps, inst["r"] if kind == icb.JOB_OC else 2.0 * inst["r"] / 1.5,
                             move=0.2, precision=icb.MIXED)
        jobs.append((cases.grid_desc(inst), kind, loop, inst["fixed"], inst["load"],
                     np.full(nel, inst["vf"])))
    for lam in rates:
        gaps = np.random.default_rng(6000 + int(lam)).exponential(1.0 / lam, len(jobs))
        srv = icb.Server(budget_bytes=150 << 30, slots=args.slots)
        t0 = time.perf_counter()
        ids, tnext = [], t0
        for j, gap in zip(jobs, gaps):
            tnext += gap
            while time.perf_counter() < tnext:
                time.sleep(min(0.002, max(0.0, tnext - time.perf_counter())))
            ids.append(srv.submit(*j))
        lat, its, ends, starts, ok = [], [], [], [], 0
        for k, jid in enumerate(ids):
            rc, info = srv.wait(jid)
            if rc == 0 and info.status == 0:
                ok += 1
                h, x, it = srv.result(jid)
                if k in first:  # the same job at an earlier rate
                    same_all = same_all and np.array_equal(h, first[k][0]) and np.array_equal(x, first[k][1])
                else:
                    first[k] = (h, x)
                lat.append(info.end_s - info.submit_s)
                its.extend(it.tolist())
                ends.append(info.end_s)
                starts.append(info.submit_s)
                if probe is None and jobs[k][1] == icb.JOB_OC:
                    probe = (jobs[k], h, x)
            srv.forget(jid)
        srv.close()
        span = max(ends) - min(starts) if ends else float("nan")
        out[str(lam)] = {"jobs": len(jobs), "completed": ok, "jobs_per_s": ok / span,
                         "job_latency_s": {"p50": float(np.median(lat)), "p99": float(np.quantile(lat, 0.99))},
                         "iter_latency_ms": {"p50": 1e3 * float(np.median(its)),
                                             "p99": 1e3 * float(np.quantile(its, 0.99))}}
        print(json.dumps({"rate": lam, **out[str(lam)]}), file=sys.stderr, flush=True)
    alone_equal = None
    if probe is not None:
        srv = icb.Server(budget_bytes=150 << 30, slots=1)
        jid = srv.submit(*probe[0])
        srv.wait(jid)
        h, x, _ = srv.result(jid)
        srv.close()
        alone_equal = bool(np.array_equal(h, probe[1]) and np.array_equal(x, probe[2]))
    best = max(out.values(), key=lambda v: v["jobs_per_s"])
    print(json.dumps({"metric": "served jobs/s (c5 Poisson mix, 150 GB admission budget)",
                      "value": best["jobs_per_s"], "unit": "jobs/s", "n_gpus": 1, "higher_is_better": True,
                      "dtype": "f64 Krylov / f32 multigrid", "data": "synthetic (seeded job stream)",
                      "config": {"workload": "70% 2D Q4 OC nelx 64-1024 aspect 2:1, 30% 3D Hex8 MMA nelx 32-128",
                                 "jobs_per_rate": args.jobs_per_rate, "iter_scale": args.iter_scale,
                                 "slots": args.slots},
                      "rates": out, "alone_vs_mixed_bitwise_equal": alone_equal,
                      "same_results_at_every_rate": same_all}), flush=True)
    return 0


def workload_solve(args):
    """One solve on the c3 geometry (half-MBB, seeded smooth densities), for
    profiling: a warm-up solve that builds the hierarchy, then the timed one.
    --size sets the grid (default 384 128 128), --solver fp64_jacobi |
    fp64_gmg | mixed_gmg (default mixed_gmg), --tc 1 puts the mixed
    V-cycle's fine-level operator on the tensor cores."""
    import numpy as np
    import cases
    import icarat_b200 as icb
    n = tuple(args.size) if args.size else (384, 128, 128)
    prec, pc = {"fp64_jacobi": (icb.FP64, icb.JACOBI), "fp64_gmg": (icb.FP64, icb.GMG),
                "mixed_gmg": (icb.MIXED, icb.GMG),
                "mixed_refine": (icb.MIXED_REFINE, icb.GMG)}[args.solver]
    ctx = icb.Context(0)
    icb.set_option("tc_operator", args.tc)
    g = cases.build_gpu(ctx, "halfmbb3d", *n)
    g.set_density(smooth_field(*n, seed=SEED))
    icb.set_option("hex8_pair", args.pair)
    mg = {"mg_smooth": args.smooth, "mg_coarse_dofs": args.coarse_dofs}
    g.solve(precision=prec, precond=pc, tol=TOL, maxit=200000, inner_tol=args.inner_tol, **mg)
    times, inf = [], None
    for _ in range(args.repeat):
        t0 = time.perf_counter()
        inf = g.solve(precision=prec, precond=pc, tol=TOL, maxit=200000, inner_tol=args.inner_tol,
                      **mg)
        times.append(time.perf_counter() - t0)
    print(json.dumps({"metric": "solve time", "value": 1e3 * min(times), "unit": "ms",
                      "all_ms": [1e3 * t for t in times], "solver": args.solver,
                      "tc_operator": args.tc, "hex8_pair": args.pair, "inner_tol": args.inner_tol,
                      "mg_smooth": args.smooth, "mg_coarse_dofs": args.coarse_dofs,
                      "tc_timeouts": icb.get_option("tc_timeouts"),
                      "config": {"workload": f"halfmbb3d {n[0]}x{n[1]}x{n[2]}", "dof": g.neq},
                      "iters": inf["iters"], "outer": inf["outer"], "matvecs": inf["matvecs"],
                      "true_relres": inf["true_relres"]}), flush=True)
    g.close()
    ctx.close()
    return 0


def profile_operator(args):
    """Set up the bench problem and launch each operator variant 3 times (for
    an ncu capture of k_matvec_h8 on the full workload; no timing printed)."""
    import torch
    import cases
    import icarat_b200 as icb
    ctx = icb.Context(0)
    kind, n = WORKLOAD
    prob = cases.build_gpu(ctx, kind, *n)
    prob.set_density(cases.uniform_density(prob.nel, SEED))
    nsoa = prob.soa_length()
    for prec, dt in ((icb.FP64, torch.float64), (icb.MIXED, torch.float32)):
        x = torch.randn(nsoa, dtype=dt, device="cuda")
        y = torch.empty_like(x)
        for _ in range(3):
            prob.operator_apply_device(x.data_ptr(), y.data_ptr(), prec)
    ctx.synchronize()
    print("profile-operator done")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline sample")
    ap.add_argument("--profile-operator", action="store_true",
                    help="only launch the operator kernels on the bench problem (for ncu)")
    ap.add_argument("--workload", default="headline",
                    choices=["headline", "c2", "c1", "c3", "batched", "serving", "operator", "solve"],
                    help="headline (default): the c3 bench line; c2: the FP64 Jacobi-PCG drop-in on "
                         "192x64x64 (both arms); the others print their own line")
    ap.add_argument("--size", type=int, nargs="+", default=None, help="c3 / operator grid override")
    ap.add_argument("--mma-steps", type=int, default=20)
    ap.add_argument("--host-loops", action="store_true",
                    help="run the multigrid PCG and OC loops as host-polled graph batches "
                         "(icb option device_loops = 0), so a profiler sees every kernel")
    ap.add_argument("--loop-only", action="store_true",
                    help="c3: only the MMA loop (no initial-design solves, no CPU sample)")
    ap.add_argument("--tc", type=int, default=0, choices=[0, 1],
                    help="solve workload: fine-level V-cycle operator on the tensor cores")
    ap.add_argument("--solver", default="mixed_gmg",
                    choices=["fp64_jacobi", "fp64_gmg", "mixed_gmg", "mixed_refine"],
                    help="solve workload: which solver")
    ap.add_argument("--pair", type=int, default=0, choices=[0, 1],
                    help="solve workload: FP32 Hex8 operator with two element rows per thread "
                         "(the library default is the one-row kernel)")
    ap.add_argument("--inner-tol", type=float, default=0.0,
                    help="solve workload, mixed_refine: inner relative tolerance (0: default)")
    ap.add_argument("--repeat", type=int, default=3, help="solve workload: timed solves")
    ap.add_argument("--smooth", type=int, default=0,
                    help="solve workload: Chebyshev steps before and after (0: the default, 2)")
    ap.add_argument("--coarse-dofs", type=int, default=0,
                    help="solve workload: coarsest-level DOF bound (0: the default, 160)")
    ap.add_argument("--instances", type=int, default=256)
    ap.add_argument("--loop-steps", type=int, default=100, help="batched: OC steps per instance")
    ap.add_argument("--batch-modes", nargs="+", default=["none"],
                    help="batched: extra comparison modes besides sequential and fused")
    ap.add_argument("--loop-steps-short", type=int, default=10,
                    help="batched: OC steps of the sequential / streams / fused comparison")
    ap.add_argument("--workers", type=int, nargs="+", default=[1, 8, 16], help="batched: host workers")
    ap.add_argument("--rates", type=float, nargs="+", default=[10, 20, 50, 100, 200, 500])
    ap.add_argument("--jobs-per-rate", type=int, default=24)
    ap.add_argument("--iter-scale", type=float, default=0.2, help="serving: scale on U[50,200] steps")
    ap.add_argument("--slots", type=int, default=8)
    ap.add_argument("--handoff", type=int, default=0,
                    help="batched: designs left when the fused solves hand them to their own "
                         "loops (0: the library default)")
    ap.add_argument("--max-connections", type=int, default=32,
                    help="batched / serving: CUDA_DEVICE_MAX_CONNECTIONS (hardware work queues "
                         "the many per-instance streams map onto; CUDA's default is 8)")
    args = ap.parse_args()
    if args.workload in ("batched", "serving") and "CUDA_DEVICE_MAX_CONNECTIONS" not in os.environ:
        # read by CUDA when the context is created, which has not happened yet
        os.environ["CUDA_DEVICE_MAX_CONNECTIONS"] = str(args.max_connections)
    if args.host_loops and args.impl == "ours":
        import icarat_b200 as icb
        icb.set_option("device_loops", 0)
    if args.profile_operator:
        return profile_operator(args)
    if args.workload == "headline":
        return headline_reference(args) if args.impl == "reference" else headline_ours(args)
    if args.workload != "c2" and args.impl == "ours":
        return {"c1": workload_c1, "c3": workload_c3, "batched": workload_batched,
                "serving": workload_serving, "operator": workload_operator,
                "solve": workload_solve}[args.workload](args)
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
