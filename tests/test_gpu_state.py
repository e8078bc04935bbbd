"""Integrator state on the GPU: checkpoint / restart, step-sequence replay,
frame output, and the failure paths, through the C ABI.

Tolerances:
  restart from a checkpoint            bit for bit (state and counters)
  a run replaying its own recorded steps  max|dm| <= 1e-9 (order-change
      rescale factors are re-derived from the recorded h, equal to ~1 ulp)
Failure paths are made on the host (a NaN planted in y0, an RHS failure
injected before any launch, a control-op bound set low): no kernel faults.
"""
import numpy as np
import pytest

import llg

pytestmark = pytest.mark.gpu


def _hole(ng=96, ny=48, prec=llg.DEMAG_FP64, alpha=0.02, strength=4.0, seed=12345):
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                         ic_jitter_eps=0.01, init_random_seed=seed)
    geo = llg.build_geometry(g)
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=strength, alpha=alpha,
                           norm_kind=llg.NORM_REG, demag_precision=prec)
    return p, geo


def _ctx(p, geo):
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    return ctx


def _run(torch, ctx, k0, k1, yout):
    for k in range(k0, k1 + 1):
        ctx.integrate(0.1 * k, yout)
    torch.cuda.synchronize()
    return yout.cpu().numpy().copy()


COUNTERS = ("nst", "nfe", "nsetups", "nni", "ncfn", "netf", "nli", "nlcf", "njvevals", "npsolves", "npe", "qlast",
            "qcur", "hlast", "hcur", "tcur")


@pytest.mark.parametrize("prec", [llg.DEMAG_FP64, llg.DEMAG_MIXED])
@pytest.mark.parametrize("via_file", [False, True])
def test_checkpoint_restart_is_bit_exact(gpu, tmp_path, prec, via_file):
    import torch
    p, geo = _hole(prec=prec)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    a = _ctx(p, geo)
    a.integrator_init(0.0, y0, llg.default_solver_opts())
    ya = torch.zeros_like(y0)
    _run(torch, a, 1, 10, ya)
    if via_file:
        path = tmp_path / "state.ckpt"
        a.write_checkpoint(str(path))
        blob = np.fromfile(str(path), dtype=np.uint8)
    else:
        blob = a.checkpoint()
    info = llg.checkpoint_inspect(blob)
    assert info.ng == p.ng and abs(info.tn - a.stats()["tcur"]) == 0.0 and info.nst == a.stats()["nst"]
    full = _run(torch, a, 11, 20, ya)
    b = _ctx(p, geo)
    if via_file:
        b.read_checkpoint(str(path))
    else:
        b.restore(blob)
    yb = torch.zeros_like(y0)
    rest = _run(torch, b, 11, 20, yb)
    sa, sb = a.stats(), b.stats()
    assert np.array_equal(full, rest), np.abs(full - rest).max()
    for k in COUNTERS:
        assert sa[k] == sb[k], k


def test_checkpoint_load_rejects_corrupt_and_foreign_blobs(gpu):
    import torch
    p, geo = _hole()
    y0 = torch.from_numpy(geo["y0"]).cuda()
    a = _ctx(p, geo)
    a.integrator_init(0.0, y0, llg.default_solver_opts())
    _run(torch, a, 1, 3, torch.zeros_like(y0))
    blob = a.checkpoint()
    bad = blob.copy()
    bad[len(bad) // 2] ^= 0x40
    with pytest.raises(llg.LLGError, match="checksum"):
        a.restore(bad)
    with pytest.raises(llg.LLGError, match="truncated"):
        a.restore(blob[:-8])
    p2, geo2 = _hole(ng=64)
    with pytest.raises(llg.LLGError, match="grid"):
        _ctx(p2, geo2).restore(blob)
    p3, _ = _hole(strength=3.0)
    with pytest.raises(llg.LLGError, match="physics"):
        _ctx(p3, geo).restore(blob)


def test_replay_of_own_steps_reproduces_the_run(gpu):
    """alpha 0.2 (the relaxation is stable): a run that replays the steps it
    recorded ends where it ended, and the replay overrides no error test."""
    import torch
    p, geo = _hole(alpha=0.2)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    a = _ctx(p, geo)
    a.integrator_init(0.0, y0, llg.default_solver_opts())
    a.record_steps(100000)
    ya = _run(torch, a, 1, 20, torch.zeros_like(y0))
    h, q = a.recorded_steps()
    assert len(h) == a.stats()["nst"] and q[0] == 1 and q.max() > 1
    b = _ctx(p, geo)
    b.integrator_init(0.0, y0, llg.default_solver_opts())
    b.replay_steps(h, q)
    yb = _run(torch, b, 1, 20, torch.zeros_like(y0))
    st = b.replay_status()
    assert st["position"] == len(h) and st["forced_accepts"] == 0
    assert np.abs(ya - yb).max() <= 1e-9
    # a replay needing more steps than were recorded stops with LLG_ERR_STATE
    c = _ctx(p, geo)
    c.integrator_init(0.0, y0, llg.default_solver_opts())
    c.replay_steps(h[:5], q[:5])
    with pytest.raises(llg.LLGError, match="LLG_ERR_STATE"):
        _run(torch, c, 1, 20, torch.zeros_like(y0))


def test_frame_from_device_matches_host_writer(gpu, tmp_path):
    import torch
    p, geo = _hole(ng=24, ny=12)
    ctx = _ctx(p, geo)
    y = torch.from_numpy(geo["y0"]).cuda()
    ctx.write_frame(str(tmp_path / "a.txt"), 0.5, y, append=False, style=llg.FRAME_FINAL)
    llg.write_frame(str(tmp_path / "b.txt"), 0.5, 24, 12, geo["y0"], append=False, style=llg.FRAME_FINAL)
    assert (tmp_path / "a.txt").read_bytes() == (tmp_path / "b.txt").read_bytes()


def test_nan_state_returns_bad_state(gpu):
    """CVODE's pre-step check on ||y||_WRMS: a NaN in y0 ends the call with
    CV_BAD_STATE (the oracle gives the same code)."""
    import torch
    p, geo = _hole()
    y0 = geo["y0"].copy()
    y0[7] = np.nan
    ctx = _ctx(p, geo)
    ctx.integrator_init(0.0, torch.from_numpy(y0).cuda(), llg.default_solver_opts())
    with pytest.raises(llg.LLGError, match="CV_BAD_STATE"):
        ctx.integrate(0.1, torch.zeros(y0.size, dtype=torch.float64, device="cuda"))


@pytest.mark.parametrize("after", [0, 25])
def test_injected_rhs_failure_propagates(gpu, after):
    """An RHS evaluation that fails (injected on the host: nothing launched)
    ends llg_integrate with CV_RHSFUNC_FAIL, as CVODE reports a callback
    returning -1; the CUDA context stays usable."""
    import torch
    p, geo = _hole()
    ctx = _ctx(p, geo)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, llg.default_solver_opts())
    ctx.inject_rhs_failure(after)
    yout = torch.zeros_like(y0)
    with pytest.raises(llg.LLGError, match="CV_RHSFUNC_FAIL"):
        for k in range(1, 40):
            ctx.integrate(0.1 * k, yout)
    assert ctx.stats()["nfe"] >= after
    ctx.inject_rhs_failure(-1)
    torch.cuda.synchronize()
    ydot = torch.zeros_like(y0)
    ctx.rhs(0.0, y0.clone(), ydot)   # the device still runs kernels
    torch.cuda.synchronize()
    assert torch.isfinite(ydot).all()


def test_device_resident_control_bound_returns_timeout(gpu):
    """The device-resident integrator counts its control operations; with a
    bound of 40 per call the step graph's loops all exit and the call returns
    LLG_ERR_TIMEOUT instead of spinning; the context then runs kernels again."""
    import torch
    p, geo = _hole()
    ctx = _ctx(p, geo)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, llg.default_solver_opts(device_resident=1))
    yout = torch.zeros_like(y0)
    ctx.integrate(0.1, yout)            # the first call starts on the host path
    ctx.set_control_op_limit(40)
    with pytest.raises(llg.LLGError, match="LLG_ERR_TIMEOUT"):
        ctx.integrate(5.0, yout)
    torch.cuda.synchronize()
    ydot = torch.zeros_like(y0)
    ctx.rhs(0.0, y0.clone(), ydot)
    torch.cuda.synchronize()
    assert torch.isfinite(ydot).all()


def test_replayed_mixed_form_within_1e4_of_fp64(gpu):
    """The mixed-precision form's own error on a hole + open-demag film
    (256x128, strength 1, alpha 0.2, t 0 -> 10 at rtol 1e-4): both forms take
    plain FP64's recorded steps, so max|dm| measures the reduced-precision
    demag alone, and an FP64 control with the demag strength changed by 1e-9
    (same steps) measures how much the film amplifies a perturbation.  This
    film relaxes without forming domains: the control stays below 1e-7 and
    the form within 1e-4 of FP64 at every output.  (At strength 4 the film
    breaks into domains near t = 4 and the 1e-9 control itself jumps to
    1e-4 there, as does the form: there the distance is the film's, not the
    form's.)"""
    import torch
    t_out = [float(t) for t in range(1, 11)]

    def run(prec, replay=None, strength=1.0):
        p, geo = _hole(256, 128, prec=prec, alpha=0.2, strength=strength)
        ctx = _ctx(p, geo)
        y0 = torch.from_numpy(geo["y0"]).cuda()
        ctx.integrator_init(0.0, y0, llg.default_solver_opts())
        if replay is None:
            ctx.record_steps(1_000_000)
        else:
            ctx.replay_steps(*replay)
        yout = torch.zeros_like(y0)
        outs = []
        for k in range(1, 101):
            ctx.integrate(0.1 * k, yout)
            if k % 10 == 0:
                torch.cuda.synchronize()
                outs.append(yout.cpu().numpy().copy())
        return outs, (ctx.recorded_steps() if replay is None else ctx.replay_status())

    a, steps = run(llg.DEMAG_FP64)
    b, st = run(llg.DEMAG_MIXED, replay=steps)
    c, _ = run(llg.DEMAG_FP64, replay=steps, strength=1.0 * (1.0 + 1e-9))
    assert st["position"] == len(steps[0])
    dms = [float(np.abs(x - y).max()) for x, y in zip(a, b)]
    dcs = [float(np.abs(x - y).max()) for x, y in zip(a, c)]
    for t, dm, dc in zip(t_out, dms, dcs):
        print(f"t={t}: replayed mixed vs FP64 max|dm| = {dm:.3e}, FP64 control {dc:.3e}")
    assert max(dcs) <= 1e-7
    assert max(dms) <= 1e-4


def test_fp32_krylov_basis_tracks_fp64_basis(gpu):
    """LLG_KRYLOV_FP32 stores the SPGMR basis in FP32 (products and sums in
    FP64).  On the stable hole + open-demag film, replaying the FP64-basis
    run's steps, the final states agree to far below the integration
    tolerance and GMRES needs about as many iterations per Newton
    iteration.  Unsupported combinations are refused."""
    import torch
    p, geo = _hole(alpha=0.2, prec=llg.DEMAG_MIXED)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    a = _ctx(p, geo)
    a.integrator_init(0.0, y0, llg.default_solver_opts())
    a.record_steps(100000)
    ya = _run(torch, a, 1, 20, torch.zeros_like(y0))
    h, q = a.recorded_steps()
    b = _ctx(p, geo)
    b.integrator_init(0.0, y0, llg.default_solver_opts(krylov_precision=llg.KRYLOV_FP32))
    b.replay_steps(h, q)
    yb = _run(torch, b, 1, 20, torch.zeros_like(y0))
    sa, sb = a.stats(), b.stats()
    dm = float(np.abs(ya - yb).max())
    ia, ib = sa["nli"] / sa["nni"], sb["nli"] / sb["nni"]
    print(f"FP32 vs FP64 Krylov basis: max|dm| {dm:.2e}, GMRES/Newton {ia:.3f} vs {ib:.3f}")
    assert dm <= 1e-6
    assert abs(ib - ia) <= 0.05 * ia + 0.05
    # its own step selection also works
    c = _ctx(p, geo)
    c.integrator_init(0.0, y0, llg.default_solver_opts(krylov_precision=llg.KRYLOV_FP32))
    yc = _run(torch, c, 1, 20, torch.zeros_like(y0))
    assert np.isfinite(yc).all() and float(np.abs(yc - ya).max()) <= 1e-3
    with pytest.raises(llg.LLGError, match="LLG_ERR_NOTSUP|failed with status -105"):
        _ctx(p, geo).integrator_init(0.0, y0, llg.default_solver_opts(krylov_precision=llg.KRYLOV_FP32,
                                                                      gs_type=llg.GS_MODIFIED))


def test_fp32_basis_with_an_inactive_learned_preconditioner_is_block_jacobi(gpu):
    """LLG_PREC_LEARNED with LLG_KRYLOV_FP32 keeps the FP64 basis while the
    network runs and hands over to block-Jacobi on the FP32 basis once it is
    off.  A learned context without weights is off from the first step, so
    its run must equal the block-Jacobi FP32-basis run bit for bit, with the
    same counters."""
    import torch
    p, geo = _hole(alpha=0.2, prec=llg.DEMAG_MIXED)
    pl = llg.default_params(p.ng, p.ny, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, alpha=0.2,
                            norm_kind=llg.NORM_REG, demag_precision=llg.DEMAG_MIXED, precond_kind=llg.PREC_LEARNED)
    y0 = torch.from_numpy(geo["y0"]).cuda()
    opts = llg.default_solver_opts(krylov_precision=llg.KRYLOV_FP32)
    out = []
    for pp in (p, pl):
        c = _ctx(pp, geo)
        c.integrator_init(0.0, y0, opts)
        out.append((_run(torch, c, 1, 10, torch.zeros_like(y0)), c.stats()))
        c.close()
    (ya, sa), (yb, sb) = out
    print("block-Jacobi", sa, "learned (no weights)", sb)
    assert np.array_equal(ya, yb)
    for k in COUNTERS:
        assert sa[k] == sb[k], k
