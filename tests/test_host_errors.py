"""Host-side error paths of the C ABI that need no GPU.

A server whose workers cannot open their device fails every job it admits
(no admitted job waits for ever), bad jobs are refused at submission, and the
batch runner checks its arguments.  Device 99 exists on no machine, so these
tests run the same with or without a GPU and launch nothing.
"""
import ctypes as C

import numpy as np
import pytest

import cases
import icarat_b200 as icb

NO_DEVICE = 99
JOB_DONE = 2  # ICB_JOB_DONE
BAD_ARG, TIMEOUT, REJECTED = -1, -5, -9


def _job():
    inst = cases.random_instance2d(np.random.default_rng(3), nelx_range=(16, 24))
    loop = icb.loop_opts(4, inst["r"], move=0.2)
    rho0 = np.full(inst["nx"] * inst["ny"], inst["vf"])
    return cases.grid_desc(inst), loop, inst["fixed"], inst["load"], rho0


def test_context_on_a_missing_device_is_an_error():
    with pytest.raises(icb.IcbError) as e:
        icb.Context(NO_DEVICE)
    assert e.value.code in (BAD_ARG, -7)  # no such device / no CUDA driver


def test_server_without_a_device_fails_every_job():
    grid, loop, fixed, load, rho0 = _job()
    s = icb.Server(device=NO_DEVICE, budget_bytes=1 << 40, slots=2)
    try:
        with pytest.raises(icb.IcbError) as e:
            s.submit(grid, 7, loop, fixed, load, rho0)  # neither OC nor MMA
        assert e.value.code == BAD_ARG
        ids = [s.submit(grid, icb.JOB_OC, loop, fixed, load, rho0) for _ in range(3)]
        for j in ids:
            rc, info = s.wait(j, timeout=60.0)
            assert rc not in (0, TIMEOUT), rc
            assert info.state == JOB_DONE and info.status == rc
    finally:
        s.close()


def test_server_rejects_a_job_over_its_budget():
    grid, loop, fixed, load, rho0 = _job()
    s = icb.Server(device=NO_DEVICE, budget_bytes=1 << 20, slots=1)
    try:
        with pytest.raises(icb.IcbError) as e:
            s.submit(grid, icb.JOB_OC, loop, fixed, load, rho0)
        assert e.value.code == REJECTED
    finally:
        s.close()


def test_server_and_batch_arguments():
    L = icb.lib()
    h = C.c_void_p()
    assert L.icb_server_create(0, 1 << 30, 0, C.byref(h)) == BAD_ARG
    assert L.icb_server_create(0, 0, 1, C.byref(h)) == BAD_ARG
    assert L.icb_run_batch(-1, None, None, None, None, None, None, 1, None) == BAD_ARG
    assert L.icb_server_destroy(None) == 0
