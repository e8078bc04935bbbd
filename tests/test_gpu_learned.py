"""Learned preconditioner on the GPU, through the C ABI.

1. The CUDA training kernels (forward, loss, backward) against the FP64
   restatement oracle/learned_ref.py (itself pinned to finite differences in
   tests/test_learned_oracle.py).  FP32 kernels vs FP64: rel 1e-4.
2. Harvest -> train -> integrate: the network is trained on the solver's own
   SPGMR solutions of a square-hole + open-demag film and then used as the
   left preconditioner; it must lower the GMRES iterations per Newton
   iteration against block-Jacobi on a fresh run of the same physics.
"""
import os
import sys

import numpy as np
import pytest

import llg
from conftest import REPO

sys.path.insert(0, os.path.join(REPO, "oracle"))
import learned_ref as L  # noqa: E402

pytestmark = pytest.mark.gpu


def test_training_kernels_match_fp64_oracle(gpu):
    rng = np.random.default_rng(3)
    theta = (rng.standard_normal(L.nparams()) * 0.1).astype(np.float32)
    nb, P = 3, 20
    batch = L.random_batch(rng, nb, P, P)
    for s in batch:   # FP32-representable inputs for both sides
        for k in ("u", "m", "mask", "ewt", "x"):
            s[k] = s[k].astype(np.float32).astype(np.float64)
        s["gamma"] = float(np.float32(s["gamma"]))
    loss_ref, g_ref = L.loss_and_grad(theta.astype(np.float64), batch)
    st = lambda k: np.stack([s[k] for s in batch])  # noqa: E731
    loss, g, z = llg.learned_loss_grad(theta, st("u"), st("m"), st("mask"), st("ewt"), st("x"),
                                       np.array([s["gamma"] for s in batch]))
    z_ref = np.stack([L.forward(theta.astype(np.float64), s["u"], s["m"], s["mask"], s["gamma"])[0]
                      for s in batch])
    print("loss", loss, loss_ref, "grad rel", np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref))
    assert abs(loss - loss_ref) <= 1e-5 * abs(loss_ref)
    assert np.linalg.norm(g - g_ref) <= 1e-4 * np.linalg.norm(g_ref)
    assert np.abs(z - z_ref).max() <= 1e-4 * np.abs(z_ref).max()


def _film(ng, ny, precond):
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, norm_kind=llg.NORM_REG,
                           precond_kind=precond)
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125, ic_jitter_eps=0.01)
    return p, llg.build_geometry(g)


def _integrate(torch, ctx, geo, t_end, opts):
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, opts)
    yout = torch.zeros_like(y0)
    for k in range(1, int(round(t_end / 0.1)) + 1):
        ctx.integrate(0.1 * k, yout)
    torch.cuda.synchronize()
    return yout.cpu().numpy(), ctx.stats()


def test_trained_network_lowers_gmres_iterations(gpu):
    import torch
    ng, ny = 192, 128
    opts = llg.default_solver_opts()
    # harvest training pairs from a block-Jacobi run
    p, geo = _film(ng, ny, llg.PREC_BLOCK_JACOBI)
    act = np.tile(geo["active"].astype(np.float64), 3)
    ch = llg.Context(p)
    ch.set_mask(act)
    ch.learned_harvest(48, 1)
    _integrate(torch, ch, geo, 1.0, opts)
    assert ch.learned_num_samples() > 8
    l0, l1 = ch.learned_train(iters=600, batch=16, patch=32, seed=5, lr=3e-3, init_scale=0.05)
    w = ch.learned_get_weights()
    print(f"training loss {l0:.4e} -> {l1:.4e} on {ch.learned_num_samples()} harvested solves")
    assert l1 < l0
    # fresh runs of the same physics, block-Jacobi vs learned
    _, base = _integrate(torch, _ctx(llg.PREC_BLOCK_JACOBI, ng, ny, act), geo, 2.0, opts)
    cl = _ctx(llg.PREC_LEARNED, ng, ny, act)
    cl.learned_set_weights(w)
    cl.learned_set_policy(False)   # learned on every solve: the network's own effect
    _, lrn = _integrate(torch, cl, geo, 2.0, opts)
    status = cl.learned_status()
    it_b = base["nli"] / base["nni"]
    it_l = lrn["nli"] / lrn["nni"]
    print(f"GMRES iterations per Newton iteration: block-Jacobi {it_b:.3f} ({base}), learned {it_l:.3f} "
          f"({lrn}), status {status}")
    assert status["active"] == 1 and status["fell_back"] == 0 and status["napply"] > 0
    assert it_l < it_b


def _ctx(precond, ng, ny, act):
    p, _ = _film(ng, ny, precond)
    c = llg.Context(p)
    c.set_mask(act)
    return c


@pytest.mark.parametrize("ng,ny", [(70, 45), (96, 64)])
def test_inference_paths_match_fp64_oracle(gpu, ng, ny):
    """Fused tensor-core inference (BF16 activations) and the layer-by-layer
    FP32 path against the FP64 network with the same BF16-rounded weights,
    on a grid that is not a multiple of the 32x16 tile, with a hole."""
    import torch
    rng = np.random.default_rng(17)
    theta = (rng.standard_normal(L.nparams()) * 0.15).astype(np.float32)
    # BF16 rounding (round to nearest even on the upper 16 bits)
    bits = theta.view(np.uint32).astype(np.uint64)
    bits = ((bits + 0x7FFF + ((bits >> 16) & 1)) >> 16) << 16
    theta_bf = bits.astype(np.uint32).view(np.float32).astype(np.float64)
    n = ng * ny
    mask = np.ones((ny, ng))
    mask[ny // 3: ny // 3 + 9, ng // 2: ng // 2 + 13] = 0.0
    z = rng.standard_normal((3, ny, ng)) * mask[None]
    m = rng.standard_normal((3, ny, ng))
    m /= np.linalg.norm(m, axis=0, keepdims=True)
    ewt = rng.uniform(0.5, 2.0, (3, ny, ng))
    gamma = 0.03
    zr, _ = L.forward(theta_bf, z, m, mask, gamma)
    ref = (ewt * zr).ravel()
    corr = np.abs(ref - (ewt * z * mask[None]).ravel()).max()
    p = llg.default_params(ng, ny, precond_kind=llg.PREC_LEARNED)
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(mask.ravel(), 3))
    ctx.learned_set_weights(theta)
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a.ravel())).cuda()  # noqa: E731
    dz, dm, de = d(z), d(m), d(ewt)
    outs = {}
    for fused in (1, 0):
        ctx.learned_set_fused(fused)
        o = torch.zeros(3 * n, dtype=torch.float64, device="cuda")
        n2 = ctx.learned_apply(dz, dm, de, gamma, o)
        outs[fused] = (o.cpu().numpy(), n2)
    ef = np.abs(outs[1][0] - ref).max() / corr
    er = np.abs(outs[0][0] - ref).max() / corr
    print(f"{ng}x{ny}: fused (BF16 activations) {ef:.2e}, FP32 layers {er:.2e} of max |correction| {corr:.3e}")
    assert er <= 1e-5
    assert ef <= 3e-2
    assert abs(outs[1][1] - np.sum(outs[1][0] ** 2)) <= 1e-10 * outs[1][1]


def test_cost_aware_policy_judges_on_the_same_trajectory(gpu):
    """Default policy: every 8th solve is a block-Jacobi probe on the same
    trajectory; the judgement (iterations of both, cost ratio kappa) is
    recorded and the context keeps the learned path only if it pays."""
    import torch
    ng, ny = 192, 128
    opts = llg.default_solver_opts()
    p, geo = _film(ng, ny, llg.PREC_BLOCK_JACOBI)
    act = np.tile(geo["active"].astype(np.float64), 3)
    ch = _ctx(llg.PREC_BLOCK_JACOBI, ng, ny, act)
    ch.learned_harvest(32, 1)
    _integrate(torch, ch, geo, 0.6, opts)
    ch.learned_train(iters=300, batch=16, patch=32, seed=5, lr=3e-3, init_scale=0.05)
    cl = _ctx(llg.PREC_LEARNED, ng, ny, act)
    cl.learned_set_weights(ch.learned_get_weights())
    _integrate(torch, cl, geo, 2.0, opts)
    st = cl.learned_status()
    print("policy", st)
    assert st["kappa"] > 0.0 and st["it_learned"] > 0.0 and st["it_block_jacobi"] > 0.0
    pays = st["it_learned"] * 1.6 + (st["it_learned"] + 1.0) * st["kappa"] < st["it_block_jacobi"] * 1.6
    assert st["fell_back"] == (0 if pays else 2)


def test_fp32_basis_takes_over_when_the_network_is_dropped(gpu):
    """LLG_KRYLOV_FP32 with the learned preconditioner: FP64 basis while the
    network runs, then (once the cost policy or a failed solve drops it)
    block-Jacobi on the FP32 basis.  An untrained network is dropped; the
    run then leaves the FP64-basis run of the same settings (the FP32 basis
    took over) and, on a damped film (alpha 0.2, demag strength 1), stays
    within 1e-3 of it and of block-Jacobi FP64 over t 0 -> 2 (the bound the
    FP32-basis form meets with its own step selection)."""
    import torch
    ng, ny = 192, 128
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125, ic_jitter_eps=0.01)
    geo = llg.build_geometry(g)
    act = np.tile(geo["active"].astype(np.float64), 3)

    def ctx(precond):
        c = llg.Context(llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=1.0, alpha=0.2,
                                           norm_kind=llg.NORM_REG, precond_kind=precond))
        c.set_mask(act)
        return c

    theta = (np.random.default_rng(23).standard_normal(L.nparams()) * 0.02).astype(np.float32)
    cb = ctx(llg.PREC_BLOCK_JACOBI)
    ref, _ = _integrate(torch, cb, geo, 2.0, llg.default_solver_opts())
    cb.close()
    res = {}
    for kp in (llg.KRYLOV_FP64, llg.KRYLOV_FP32):
        c = ctx(llg.PREC_LEARNED)
        c.learned_set_weights(theta)
        y, st = _integrate(torch, c, geo, 2.0, llg.default_solver_opts(krylov_precision=kp))
        res[kp] = (y, st, c.learned_status())
        c.close()
    (y64, s64, l64), (y32, s32, l32) = res[llg.KRYLOV_FP64], res[llg.KRYLOV_FP32]
    d64, dref = float(np.abs(y32 - y64).max()), float(np.abs(y32 - ref).max())
    print("FP64 basis", s64, l64, "FP32 after the network", s32, l32, "max|dm| vs FP64 basis", d64,
          "vs block-Jacobi", dref)
    assert l32["fell_back"] != 0 and l32["napply"] > 0
    assert not np.array_equal(y32, y64)
    assert np.isfinite(y32).all() and d64 <= 1e-3 and dref <= 1e-3
