"""Many runs on one GPU: the batch runner and the continuous-batching server.

Every run is deterministic and independent: its compliance history and final
design are bitwise the same whether it runs alone, sequentially or mixed with
other jobs on other streams.
"""
import numpy as np
import pytest

import cases
import icarat_b200 as icb

pytestmark = pytest.mark.gpu


def _small_instances(n, seed):
    rng = np.random.default_rng(seed)
    return [cases.random_instance2d(rng, nelx_range=(16, 80)) for _ in range(n)]


def test_batch_equals_sequential():
    insts = _small_instances(6, 1)
    ctxs = [icb.Context(0) for _ in insts]
    probs = [cases.build_instance(c, i) for c, i in zip(ctxs, insts)]
    opts = [icb.loop_opts(8, i["r"], move=0.2) for i in insts]
    rho0 = [np.full(p.nel, i["vf"]) for p, i in zip(probs, insts)]
    h1, x1, s1 = icb.run_batch(probs, [0] * len(probs), opts, rho0, nworkers=1)
    h4, x4, s4 = icb.run_batch(probs, [0] * len(probs), opts, rho0, nworkers=4)
    assert (s1 == 0).all() and (s4 == 0).all()
    for a, b in zip(h1, h4):
        assert np.array_equal(a, b)
    for a, b in zip(x1, x4):
        assert np.array_equal(a, b)
    # and equal to the single-run entry point
    ha, xa = icb.run_loop(probs[2], "oc", rho0[2], 8, insts[2]["r"], move=0.2)
    assert np.array_equal(ha, h1[2]) and np.array_equal(xa, x1[2])


@pytest.mark.parametrize("precision", [icb.FP64, icb.MIXED])
def test_fused_batch_equals_each_problem_alone(precision):
    """icb_run_batch advances qualifying 2D OC loops together (the solves of
    every problem as one batched launch per kernel): each problem's history
    and design are bitwise those of its own icb_run_oc, also when the runs
    have different step counts (the batch shrinks as runs finish) and
    hierarchies of different depth."""
    rng = np.random.default_rng(11)
    insts = [cases.random_instance2d(rng, nelx_range=(12, 150)) for _ in range(7)]
    ctxs = [icb.Context(0) for _ in insts]
    probs = [cases.build_instance(c, i) for c, i in zip(ctxs, insts)]
    steps = [6, 4, 6, 5, 6, 3, 6]
    opts = [icb.loop_opts(k, i["r"], move=0.2, precision=precision) for k, i in zip(steps, insts)]
    rho0 = [np.full(p.nel, i["vf"]) for p, i in zip(probs, insts)]
    assert icb.get_option("batch_fused") == 1
    hf, xf, sf = icb.run_batch(probs, [0] * len(probs), opts, rho0, nworkers=1)
    assert (sf == 0).all()
    for k, (p, i) in enumerate(zip(probs, insts)):
        ha, xa = icb.run_loop(p, "oc", rho0[k], steps[k], i["r"], move=0.2, precision=precision)
        assert np.array_equal(ha, hf[k]), k
        assert np.array_equal(xa, xf[k]), k
    icb.set_option("batch_fused", 0)
    try:
        hw, xw, sw = icb.run_batch(probs, [0] * len(probs), opts, rho0, nworkers=3)
    finally:
        icb.set_option("batch_fused", 1)
    assert (sw == 0).all()
    for a, b in zip(hw + xw, hf + xf):
        assert np.array_equal(a, b)
    for p in probs:
        p.close()
    for c in ctxs:
        c.close()


@pytest.mark.parametrize("handoff", [0, 5, 1000])
def test_fused_batch_handoff_keeps_results(handoff):
    """The fused batch hands the designs still iterating to their own solve
    loops once few are left (option batch_handoff): never (0 here means the
    default rule, which hands off the last one of these seven), with five
    left, or at once (1000): each design's history and design stay bitwise
    those of its own icb_run_oc."""
    rng = np.random.default_rng(12)
    insts = [cases.random_instance2d(rng, nelx_range=(12, 120)) for _ in range(7)]
    ctxs = [icb.Context(0) for _ in insts]
    probs = [cases.build_instance(c, i) for c, i in zip(ctxs, insts)]
    steps = [4, 3, 4, 4, 2, 4, 4]
    opts = [icb.loop_opts(k, i["r"], move=0.2, precision=icb.MIXED) for k, i in zip(steps, insts)]
    rho0 = [np.full(p.nel, i["vf"]) for p, i in zip(probs, insts)]
    icb.set_option("batch_handoff", handoff)
    try:
        assert icb.get_option("batch_handoff") == handoff
        hf, xf, sf = icb.run_batch(probs, [0] * len(probs), opts, rho0, nworkers=1)
    finally:
        icb.set_option("batch_handoff", 0)
    assert (sf == 0).all()
    for k, (p, i) in enumerate(zip(probs, insts)):
        ha, xa = icb.run_loop(p, "oc", rho0[k], steps[k], i["r"], move=0.2, precision=icb.MIXED)
        assert np.array_equal(ha, hf[k]), k
        assert np.array_equal(xa, xf[k]), k
    for p in probs:
        p.close()
    for c in ctxs:
        c.close()


def _job(inst, kind, nsteps):
    loop = icb.loop_opts(nsteps, inst["r"] if kind == icb.JOB_OC else 2.0 * inst["r"] / 1.5,
                         move=0.2)
    nel = inst["nx"] * inst["ny"] * (inst["nz"] if inst["dim"] == 3 else 1)
    return (cases.grid_desc(inst), kind, loop, inst["fixed"], inst["load"], np.full(nel, inst["vf"]))


def test_server_result_same_alone_and_in_the_mix():
    rng = np.random.default_rng(5)
    a = cases.random_instance2d(rng, nelx_range=(40, 60))
    b = cases.random_instance3d(rng, nelx_range=(8, 12))
    others = [cases.random_instance2d(rng, nelx_range=(20, 90)) for _ in range(4)]
    ja, jb = _job(a, icb.JOB_OC, 12), _job(b, icb.JOB_MMA, 6)
    s1 = icb.Server(budget_bytes=8 << 30, slots=1)
    ia, ib = s1.submit(*ja), s1.submit(*jb)
    assert s1.wait(ia)[0] == 0 and s1.wait(ib)[0] == 0
    ha, xa, _ = s1.result(ia)
    hb, xb, _ = s1.result(ib)
    s1.close()
    s4 = icb.Server(budget_bytes=8 << 30, slots=4)
    ids = [s4.submit(*_job(o, icb.JOB_OC, 10)) for o in others[:2]]
    ia2 = s4.submit(*ja)
    ids += [s4.submit(*_job(o, icb.JOB_OC, 10)) for o in others[2:]]
    ib2 = s4.submit(*jb)
    infos = {}
    for j in ids + [ia2, ib2]:
        rc, inf = s4.wait(j)
        assert rc == 0
        infos[j] = inf
    ha2, xa2, ita = s4.result(ia2)
    hb2, xb2, _ = s4.result(ib2)
    assert np.array_equal(ha, ha2) and np.array_equal(xa, xa2)
    assert np.array_equal(hb, hb2) and np.array_equal(xb, xb2)
    assert (ita > 0).all()
    # jobs ran concurrently: some start before an earlier one finished
    spans = sorted((infos[j].start_s, infos[j].end_s) for j in infos)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    s4.close()


def test_server_admission_budget_and_cancel():
    rng = np.random.default_rng(9)
    big = cases.random_instance2d(rng, nelx_range=(200, 200), aspect_fixed=2.0)
    g = cases.grid_desc(big)
    fp = icb.lib().icb_job_footprint(g, icb.JOB_OC)
    assert fp > 0
    # budget for one such job at a time: both still complete, one after the other
    s = icb.Server(budget_bytes=int(fp * 1.5), slots=4)
    j1, j2 = s.submit(*_job(big, icb.JOB_OC, 4)), s.submit(*_job(big, icb.JOB_OC, 4))
    r1, i1 = s.wait(j1)
    r2, i2 = s.wait(j2)
    assert r1 == 0 and r2 == 0
    assert i2.start_s >= i1.end_s - 1e-6 or i1.start_s >= i2.end_s - 1e-6
    # a job that can never fit is rejected at submission
    huge = cases.random_instance2d(rng, nelx_range=(600, 600), aspect_fixed=1.0)
    with pytest.raises(icb.IcbError) as e:
        s.submit(*_job(huge, icb.JOB_OC, 2))
    assert e.value.code == -9
    s.close()
    # cancelling a queued job
    s = icb.Server(budget_bytes=8 << 30, slots=1)
    ja = s.submit(*_job(big, icb.JOB_OC, 6))
    jb = s.submit(*_job(big, icb.JOB_OC, 6))
    jc = s.submit(*_job(big, icb.JOB_OC, 6))
    assert s.cancel(jc) == 0
    rc, inf = s.wait(jc)
    assert inf.state == 3
    assert s.wait(ja)[0] == 0 and s.wait(jb)[0] == 0
    s.close()
