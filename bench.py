#!/usr/bin/env python
"""Benchmark of the SIMP analysis-and-sensitivity step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    (N > 1: launched by torch.distributed.run, one rank per GPU)

Workload (one step): the 192x64x64 Hex8 cantilever (2,446,275 DOF, numeq
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
    ms = e0.elapsed_time(e1)
    units = float(numeq) * mv
    if dist is not None:
        t = torch.tensor([ms], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        u = torch.tensor([units], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(u)
        ms, units = float(t.item()), float(u.item())
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
    ms2 = f0.elapsed_time(f1)
    units2 = float(numeq) * mv2
    if dist is not None:
        t = torch.tensor([ms2], device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        u = torch.tensor([units2], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(u)
        ms2, units2 = float(t.item()), float(u.item())
    e2e = {"value": units2 / (ms2 * 1e-3), "unit": UNIT,
           "h2d_bytes_per_step": 8 * prob.nel,
           "d2h_bytes_per_step": 8 * (numeq + prob.nel + 1)}

    # ---- roofline of the dominant kernel (FP64 operator), timed live
    nsoa = prob.soa_length()
    x = torch.randn(nsoa, dtype=torch.float64, device=f"cuda:{local}")
    y = torch.empty_like(x)
    prob.set_density_device(rho_d.data_ptr())
    for _ in range(5):
        prob.operator_apply_device(x.data_ptr(), y.data_ptr(), icb.FP64)
    R = 50
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    for _ in range(R):
        prob.operator_apply_device(x.data_ptr(), y.data_ptr(), icb.FP64)
    g1.record(stream)
    torch.cuda.synchronize()
    t_mv = g0.elapsed_time(g1) / R * 1e-3
    ndof = prob.neq
    alg_bytes = 8 * (2 * ndof + prob.nel)
    flops = 2 * 576 * prob.nel
    peak, peak_kind = _peaks()
    achieved = alg_bytes / t_mv / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": _traffic("matvec_fp64_cantilever3d"),
                "kernel": "k_matvec_h8<double>", "launch_us": t_mv * 1e6,
                "peak_source": peak_kind,
                "fp64_tflops": flops / t_mv / 1e12,
                "note": "FP64 element contraction: 1152 flop per element"}

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
    args = ap.parse_args()
    if args.profile_operator:
        return profile_operator(args)
    if args.impl == "reference":
        return reference_arm(args)
    return ours_arm(args)


if __name__ == "__main__":
    sys.exit(main())
