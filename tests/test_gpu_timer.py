"""Live kernel timer (llg_kernel_timer_start / _stop) on the GPU.

An event pair brackets every stride-th launch of each selected kernel family
(the 1st, (stride+1)-th, ...) on the context's stream, up to max_launches per
family.  Checks: the number of timed launches follows the stride exactly
against the library's own launch counters, the timed durations are positive,
timing changes no result, and bad arguments are refused.
"""
import ctypes as C

import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu

ARNOLDI, ROWS_FWD, COLS, ROWS_INV = 2, 6, 7, 8
LLG_ERR_ARG = -100   # include/llg.h


def _run(lib, stride, timed):
    import torch
    p = llg.default_params(96, 64, demag_mode=llg.DEMAG_OPEN, demag_strength=3.0)
    geo = llg.build_geometry(llg.default_geom(96, 64, ic_jitter_eps=0.01))
    ctx = llg.Context(p)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, llg.default_solver_opts())
    yout = torch.zeros_like(y0)
    ctx.integrate(0.1, yout)
    c0 = (C.c_int64 * 16)()
    lib.llg_kernel_counts(c0, 16)
    mask = (1 << ARNOLDI) | (1 << ROWS_FWD) | (1 << COLS) | (1 << ROWS_INV)
    if timed:
        assert lib.llg_kernel_timer_start(ctx.h, mask, 2000, stride) == 0
    for k in range(2, 8):
        ctx.integrate(0.1 * k, yout)
    tot = (C.c_double * 16)()
    nl = (C.c_int64 * 16)()
    if timed:
        assert lib.llg_kernel_timer_stop(ctx.h, tot, nl, 16) == 0
    c1 = (C.c_int64 * 16)()
    lib.llg_kernel_counts(c1, 16)
    torch.cuda.synchronize()
    y = yout.cpu().numpy()
    ctx.close()
    return y, [c1[k] - c0[k] for k in range(16)], list(tot), list(nl)


@pytest.mark.parametrize("stride", [1, 3])
def test_timer_samples_every_stride_th_launch(gpu, stride):
    lib = llg.load()
    y_plain, _, _, _ = _run(lib, stride, timed=False)
    y, launched, tot, nl = _run(lib, stride, timed=True)
    for fam in (ARNOLDI, ROWS_FWD, COLS, ROWS_INV):
        assert launched[fam] > 0, fam
        assert nl[fam] == -(-launched[fam] // stride), (fam, nl[fam], launched[fam])
        assert tot[fam] > 0.0
        assert 0.0 < tot[fam] / nl[fam] < 100.0   # ms per launch
    # the event records only end the chained launch of the kernels they bracket
    assert np.array_equal(y, y_plain)


def test_timer_rejects_bad_arguments(gpu):
    lib = llg.load()
    p = llg.default_params(64, 32)
    ctx = llg.Context(p)
    assert lib.llg_kernel_timer_start(ctx.h, 1 << ARNOLDI, 0, 1) == LLG_ERR_ARG
    assert lib.llg_kernel_timer_start(ctx.h, 1 << ARNOLDI, 10, 0) == LLG_ERR_ARG
    tot = (C.c_double * 16)()
    nl = (C.c_int64 * 16)()
    assert lib.llg_kernel_timer_stop(ctx.h, tot, nl, 16) != 0   # not started
    ctx.close()
