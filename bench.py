"""Benchmark: simulated time per wall-second of the 2-D LLG integration.

Workload (one B200, the configuration the metric is quoted on): 1536x512
cells, centred square hole of side 0.25*ny, open-boundary FFT demag
(strength 4, thickness 1, zero-padded 3072x1024 transform grid), exchange
A=1, uniaxial k=0.1 along +x, Zeeman (0,0,0.05), alpha=0.02, free edges,
uniform (1,0,0) + seeded +-0.01 jitter, BDF + Newton + SPGMR(5) with 3x3
block-Jacobi, rtol 1e-4 / atol 1e-6.  Synthetic data (seeded builders).

Timed window (both arms): a fresh instance integrated from t = 0 over K
steps of --dt simulated time (default 1.0), each step through llg_integrate
at the reference's 0.1 output cadence; value = K*dt / device time (CUDA
events on the library's stream, max over ranks).  Warm-up: W output
intervals (0.1 each) on a throwaway instance of the same form.  The state
(>= 20 vectors of 18.9 MB) exceeds L2, so no flush is needed.

Forms (--form): "plain" is the reference method in FP64; "mixed" runs the
demag transforms in reduced precision (FP32 rows, tensor-core FP16 hi+lo
column DFT stages with FP32 accumulation); "mixed32" also stores the SPGMR
basis in FP32 (the default: the fastest form measured); "learned+mixed" adds
the learned preconditioner (kept only while it pays for itself; the line
names what ran) and "learned+mixed32" does the same with block-Jacobi
continuing on the FP32 basis once the network is dropped.  By default the best form is timed, then plain FP64 the same way; the
line reports both, their ratio and the form's accuracy: max|dm| against
plain FP64 with both runs taking plain FP64's recorded step sequence
(step-sequence replay), at t = 1, 5, 20, 200.

--impl reference runs the CPU restatement of the reference path (the oracle;
the reference itself needs SUNDIALS, which is absent) on all host cores,
over the same window.  Multi-GPU: independent replicas (one instance per
rank, no collective in the hot path); only the timing max uses
torch.distributed.
"""
import argparse
import ctypes as C
import json
import os
import select
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "gpu-micromagnetics-irregular_b200")
sys.path.insert(0, PKG)
import llg  # noqa: E402

METRIC = "sim-time/wall-s @1536x512+demag, learned+mixed vs plain FP64, |Δm|≤1e-4"
UNIT = "sim-time/wall-s"
KERNEL_NAMES = ["rhs", "jtv", "arnoldi_op", "psetup", "psolve", "normalize", "demag_rows_fwd",
                "demag_cols_conv", "demag_rows_inv", "reduce", "elementwise", "learned", "other"]
TIMED_FAMILIES = (2, 6, 7, 8)   # Arnoldi operator, demag rows forward / columns / rows inverse
TIMER_STRIDE = 7                # event pair around every 7th launch of a family (odd: both Arnoldi
                                # launches of a solve are sampled); the rest keep their chained launch


# Gram-Schmidt for every form: CVODE's classical Gram-Schmidt with its
# reorthogonalisation test (one extra pass when the new vector loses 3 digits),
# which needs one read-back per Arnoldi iteration.  The reference lets SPGMR
# pick modified Gram-Schmidt at neq >= 5e5 (2d_i2/2d_fft.cu:674-679), a
# sequential dot-then-update chain; its plain FP64 throughput with that choice
# is measured beside the headline (plain_fp64_reference_gs_value).
GS = llg.GS_CLASSICAL
WORKLOAD = ("1536x512 cells, square hole side 0.25*ny, open FFT demag strength 4 (3072x1024 padded), "
            "A=1 k=0.1(+x) h=(0,0,0.05) alpha=0.02, free edges, rtol 1e-4 atol 1e-6, SPGMR(5), block-Jacobi")


def workload(ng=1536, ny=512, seed=12345, gs=None):
    p = llg.default_params(ng, ny, demag_mode=llg.DEMAG_OPEN, demag_strength=4.0, demag_thick=1.0,
                           bc=llg.BC_FREE, norm_kind=llg.NORM_REG)
    g = llg.default_geom(ng, ny, geometry_kind=llg.GEOM_HOLE_SQUARE, hole_radius_frac_y=0.125,
                         ic_jitter_eps=0.01, init_random_seed=seed)
    o = llg.default_solver_opts(rtol=1e-4, atol=1e-6, maxl=5, gs_type=GS if gs is None else gs)
    return p, g, o


def bench_config(args, world):
    """The workload description both arms print (identical dicts)."""
    return {"workload": WORKLOAD, "sim_time_per_step": args.dt, "output_interval": 0.1,
            "window": f"fresh instance, t 0 -> {args.steps * args.dt:g}",
            "warmup": f"{args.warmup} output intervals on a throwaway instance",
            "parallelism": f"replicas x{world}", "l2": "state > 126 MB L2 (>= 20 vectors x 18.9 MB); no flush"}


def algorithmic_bytes(kid, ng, ny, dims, mixed=False, kf32=False):
    """Compulsory HBM bytes of one launch of kernel family kid (FP64 state;
    the mixed demag chain keeps its spectra and tensor spectra in FP32; an
    FP32 Krylov basis halves V and the operator's block inverse)."""
    n = ng * ny
    px, py, hx, nrows = dims
    S = 3 * hx * nrows * (8 if mixed else 16)
    if kid == 0:   # rhs: y, hd, mask in; ydot out
        return 24 * n + 24 * n + n + 24 * n
    if kid == 1:   # jtv: y, v, mask in; Jv out
        return 24 * n + 24 * n + n + 24 * n
    if kid == 2:   # arnoldi: V_l, ewt, y, stored block inverse (9 values), mask in; V_l+1 out
        if kf32:
            return 12 * n + 24 * n + 24 * n + 36 * n + n + 12 * n
        return 3 * 24 * n + 72 * n + n + 24 * n
    if kid == 3:   # psetup: y, hd, mask in; m, h, block inverse out
        return 24 * n + 24 * n + n + 48 * n + 72 * n
    if kid == 4:   # psolve: frozen m, h, r, mask in; z out
        return 72 * n + n + 24 * n
    if kid == 6:   # rows forward: y in; row spectra out
        return 24 * n + S
    if kid == 7:   # columns: spectra in/out + tensor (xx,yy,zz real, xy complex)
        return 2 * S + hx * py * (20 if mixed else 40)
    if kid == 8:   # rows inverse: spectra in; h out
        return S + 24 * n
    if kid == 9:   # dot_multi of 6 vectors: 7 vectors read
        return 7 * 24 * n
    if kid == 10:  # linear combination of 6 vectors: 6 read + 1 write
        return 7 * 24 * n
    return 0


class Clocks:
    def __init__(self, dev):
        self.proc = None
        self.dev = dev

    def __enter__(self):
        # the sampler is started, and its first sample (taken before the timed
        # region) read and dropped, before the caller starts timing: its
        # start-up (NVML initialisation) is not part of the timed work
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            ready, _, _ = select.select([self.proc.stdout], [], [], 10.0)
            if ready:
                self.proc.stdout.readline()
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (getattr(self, "out", "") or "").splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 7:
                try:
                    rows.append((float(parts[0]), float(parts[1]), parts[3:7]))
                except ValueError:
                    pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[2]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=300))
    return world, rank, local


def dist_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def make_ctx(p, g):
    geo = llg.build_geometry(g, want=("active", "y0"))
    ctx = llg.Context(p)
    ctx.set_mask(np.tile(geo["active"].astype(np.float64), 3))
    return ctx, geo


# Forms of the same workload.  "plain" is the reference method in FP64; the
# others change only the demag transform precision and the preconditioner.
FORMS = {
    "plain": dict(demag_precision=llg.DEMAG_FP64, learned=False, name="plain FP64",
                  desc="plain FP64 (block-Jacobi, FP64 FFT demag)"),
    "mixed": dict(demag_precision=llg.DEMAG_MIXED, learned=False, name="mixed-precision demag",
                  desc="mixed-precision demag (FP32 row FFTs, tcgen05 FP16 hi+lo column DFT stages with FP32 "
                       "accumulation), block-Jacobi; FP64 state, norms, Newton update, Gram-Schmidt"),
    "mixed32": dict(demag_precision=llg.DEMAG_MIXED, learned=False, krylov=llg.KRYLOV_FP32,
                    name="mixed-precision demag + FP32 Krylov basis",
                    desc="mixed-precision demag (FP32 row FFTs, tcgen05 FP16 hi+lo column DFT stages with FP32 "
                         "accumulation) and the SPGMR Krylov basis stored in FP32 (Arnoldi operator, Gram-Schmidt "
                         "dots and update, correction read it; every product and sum in FP64), block-Jacobi; FP64 "
                         "state, norms, Newton update, Gram-Schmidt dots"),
    "learned+mixed": dict(demag_precision=llg.DEMAG_MIXED, learned=True,
                          name="learned preconditioner + mixed-precision demag",
                          desc="learned preconditioner (3-layer 3x3 conv, 16 channels, BF16 weights, FP32 "
                               "accumulation, fused tcgen05 inference, on top of block-Jacobi, trained on the GPU on "
                               "this workload's own harvested SPGMR solves; every 8th solve probes block-Jacobi and "
                               "the learned path stays only while it pays for its cost) + mixed-precision demag"),
}
FORMS["learned+mixed32"] = dict(FORMS["learned+mixed"], krylov=llg.KRYLOV_FP32,
                                name="learned preconditioner + mixed-precision demag, FP32 Krylov basis after it",
                                desc=FORMS["learned+mixed"]["desc"] + "; once the network is dropped, block-Jacobi "
                                     "continues on an FP32 Krylov basis (the mixed32 form)")
# the default (headline) form: the fastest measured at the same accuracy
# (the learned preconditioner does not pay on this workload: its cost test
# drops it after 55 applications; the learned forms are timed beside it)
BEST_FORM = "mixed32"
TRAIN = dict(t_harvest=1.0, max_samples=32, stride=2, iters=600, batch=16, patch=32, seed=5, lr=3e-3,
             init_scale=0.05)
_weights_cache = {}


def train_weights(rank):
    """Harvest block-Jacobi SPGMR solves of the workload over t in [0, 1] and
    train the network on them (setup phase, outside every timed region)."""
    import torch
    if "w" in _weights_cache:
        return _weights_cache["w"], _weights_cache["info"]
    t0 = time.perf_counter()
    p, g, o = workload(seed=12345 + rank)
    p.demag_precision = llg.DEMAG_MIXED
    ctx, geo = make_ctx(p, g)
    ctx.learned_harvest(TRAIN["max_samples"], TRAIN["stride"])
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, o)
    yout = torch.zeros_like(y0)
    for k in range(1, int(round(TRAIN["t_harvest"] / 0.1)) + 1):
        ctx.integrate(0.1 * k, yout)
    t1 = time.perf_counter()
    l0, l1 = ctx.learned_train(iters=TRAIN["iters"], batch=TRAIN["batch"], patch=TRAIN["patch"],
                               seed=TRAIN["seed"], lr=TRAIN["lr"], init_scale=TRAIN["init_scale"])
    torch.cuda.synchronize()
    t2 = time.perf_counter()
    w = ctx.learned_get_weights()
    info = {"samples": ctx.learned_num_samples(), "harvest_s": t1 - t0, "train_s": t2 - t1,
            "loss_first": l0, "loss_last": l1, **{k: v for k, v in TRAIN.items()}}
    ctx.close()
    _weights_cache["w"], _weights_cache["info"] = w, info
    return w, info


def form_params(form, seed, gs=None):
    p, g, o = workload(seed=seed, gs=gs)
    o.krylov_precision = FORMS[form].get("krylov", llg.KRYLOV_FP64)
    p.demag_precision = FORMS[form]["demag_precision"]
    p.precond_kind = llg.PREC_LEARNED if FORMS[form]["learned"] else llg.PREC_BLOCK_JACOBI
    return p, g, o


def timed_run(args, form, world, rank, local, lib, clocks=True, gs=None):
    """W warm-up output intervals on a throwaway instance, then K timed steps
    of a fresh instance of `form` from t = 0."""
    import torch
    sub = max(1, int(round(args.dt / 0.1)))

    def instance():
        p, g, o = form_params(form, 12345 + rank, gs)
        ctx, geo = make_ctx(p, g)
        if FORMS[form]["learned"]:
            ctx.learned_set_weights(train_weights(rank)[0])
        y0 = torch.from_numpy(geo["y0"]).cuda()
        ctx.integrator_init(0.0, y0, o)
        return ctx, y0, p, g, o

    wctx, wy0, *_ = instance()
    wout = torch.zeros_like(wy0)
    for k in range(1, args.warmup + 1):
        wctx.integrate(0.1 * k, wout)
    torch.cuda.synchronize()
    wctx.close()
    del wctx, wy0, wout
    ctx, y0, p, g, o = instance()
    yout = torch.zeros_like(y0)
    state = {"t": 0.0}

    def step():
        for k in range(sub):
            ctx.integrate(state["t"] + args.dt * (k + 1) / sub, yout)
        state["t"] += args.dt

    counts0 = (C.c_int64 * 16)()
    counts1 = (C.c_int64 * 16)()
    lib.llg_kernel_counts(counts0, 16)
    st0 = ctx.stats()
    # live per-launch device time of the Arnoldi operator and the demag stages
    # (an event pair around every TIMER_STRIDE-th of their launches inside the
    # timed region)
    timed_mask = sum(1 << k for k in TIMED_FAMILIES)
    llg._check(lib.llg_kernel_timer_start(ctx.h, timed_mask, 20000, TIMER_STRIDE), "llg_kernel_timer_start")
    torch.cuda.synchronize()
    dist_barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clk = Clocks(local) if clocks else None
    if clk:
        clk.__enter__()
    if args.profile_window:
        torch.cuda.profiler.start()
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    if args.profile_window:
        torch.cuda.profiler.stop()
    if clk:
        clk.__exit__(None, None, None)
    ms = dist_max(e0.elapsed_time(e1), world)
    dist_barrier(world)
    tot = (C.c_double * 16)()
    nl = (C.c_int64 * 16)()
    llg._check(lib.llg_kernel_timer_stop(ctx.h, tot, nl, 16), "llg_kernel_timer_stop")
    live = {KERNEL_NAMES[k]: {"total_ms": tot[k], "launches": int(nl[k])} for k in TIMED_FAMILIES}
    lib.llg_kernel_counts(counts1, 16)
    st1 = ctx.stats()
    launches = {KERNEL_NAMES[k]: int(counts1[k] - counts0[k]) for k in range(13)}
    dst = {k: st1[k] - st0[k] for k in ("nst", "nfe", "nni", "nli", "nsetups", "netf", "ncfn")}
    ran = FORMS[form]["name"]
    if FORMS[form]["learned"]:
        ls = ctx.learned_status()
        dst["learned_status"] = ls
        if ls["fell_back"]:
            after = "mixed32" if FORMS[form].get("krylov") == llg.KRYLOV_FP32 else "mixed"
            ran = f"{FORMS[after]['name']} (learned preconditioner fell back to block-Jacobi: " + \
                  ("its cost exceeded its iteration saving" if ls["fell_back"] == 2 else "a learned solve failed") + ")"
        ran += f"; learned applications {ls['napply']}"
    return {"ctx": ctx, "p": p, "g": g, "o": o, "yout": yout, "t": state["t"], "ms": ms, "launches": launches,
            "counters": dst, "value": world * args.steps * args.dt / (ms / 1000.0), "clocks": clk, "live": live,
            "ran": ran}


def roofline_for(lib, run, ng, ny, mixed, kf32=False):
    """Roofline of the kernel with the largest live device-time share in the
    timed region: algorithmic bytes per launch / its live average launch time
    (CUDA events around each launch on the integrator's stream)."""
    live = run["live"]
    total_ms = run["ms"]
    # share of the timed region: sampled average launch time x the family's
    # launches in the region
    share = {k: v["total_ms"] / v["launches"] * run["launches"][k] / total_ms
             for k, v in live.items() if v["launches"] > 0}
    dom = max(share, key=share.get)
    kid = KERNEL_NAMES.index(dom)
    px, py = 2 * ng, 2 * ny
    dd = (px, py, px // 2 + 1, ny)
    peaks = {}
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "of measured" if "hbm_gbs" in peaks else "of fallback"
    abytes = algorithmic_bytes(kid, ng, ny, dd, mixed, kf32)
    avg_ms = live[dom]["total_ms"] / live[dom]["launches"]
    achieved = abytes / (avg_ms * 1e-3) / 1e9
    traffic = None
    try:
        with open(os.path.join(REPO, "profiles", "traffic_per_launch.json")) as f:
            traffic = json.load(f).get(("mixed32:" if kf32 else "mixed:" if mixed else "") + dom)
    except Exception:
        pass
    return {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic,
            "algorithmic_bytes_per_launch": abytes, "avg_launch_ms": avg_ms,
            "peak_source": f"{peak_src} hbm_gbs (burst copy)",
            "live_avg_launch_ms": {k: v["total_ms"] / max(v["launches"], 1) for k, v in live.items()},
            "live_launches_timed": {k: v["launches"] for k, v in live.items()},
            "live_share_of_timed_region": share,
            "timing": f"CUDA events on the integrator's stream around every {TIMER_STRIDE}th launch of these "
                      "families inside the timed region"}


def fixed_run(form, rank, t_out, strength_scale=1.0, rtol=None, record=False, replay=None):
    """Integrate a fresh instance of `form` from t=0 at the 0.1 output cadence
    and return y at each t in t_out (and the recorded steps / replay status)."""
    import torch
    p, g, o = form_params(form, 12345 + rank)
    p.demag_strength *= strength_scale
    if rtol is not None:
        o.rtol, o.atol = rtol, rtol * 1e-2
    ctx, geo = make_ctx(p, g)
    if FORMS[form]["learned"]:
        ctx.learned_set_weights(train_weights(rank)[0])
    y0 = torch.from_numpy(geo["y0"]).cuda()
    ctx.integrator_init(0.0, y0, o)
    if record:
        ctx.record_steps(10_000_000)
    if replay is not None:
        ctx.replay_steps(*replay)
    yout = torch.zeros_like(y0)
    outs = {}
    kmax = int(round(max(t_out) / 0.1))
    want = {int(round(t / 0.1)) for t in t_out}
    for k in range(1, kmax + 1):
        ctx.integrate(0.1 * k, yout)
        if k in want:
            outs[round(0.1 * k, 6)] = yout.cpu().numpy().copy()
    extra = {}
    if record:
        extra["steps"] = ctx.recorded_steps()
    if replay is not None:
        extra["replay"] = ctx.replay_status()
    if FORMS[form]["learned"]:
        extra["learned_status"] = ctx.learned_status()
    ctx.close()
    return outs, extra


def replay_accuracy(form, rank, t_out=(1.0, 5.0, 20.0, 200.0), t_floor=(1.0, 5.0)):
    """max|dm| of `form` against plain FP64 on the bench workload with both
    runs taking plain FP64's accepted step sequence (recorded, then replayed):
    what remains is the form's own arithmetic, not step selection.  Beside
    it, on the same steps, a plain FP64 run with the demag strength scaled by
    (1 + 1e-9) shows how much the workload's dynamics amplify a tiny
    perturbation; and plain FP64 at rtol 1e-6 against rtol 1e-8 shows the
    integration-error floor of a tighter tolerance."""
    md = lambda x, y, ts: [float(np.abs(x[round(t, 6)] - y[round(t, 6)]).max()) for t in ts]  # noqa: E731
    a, ra = fixed_run("plain", rank, t_out, record=True)
    steps = ra["steps"]
    b, rb = fixed_run(form, rank, t_out, replay=steps)
    c, rc = fixed_run("plain", rank, t_out, strength_scale=1.0 + 1e-9, replay=steps)
    f6, _ = fixed_run("plain", rank, t_floor, rtol=1e-6)
    f8, _ = fixed_run("plain", rank, t_floor, rtol=1e-8)
    dm = md(b, a, t_out)
    ok_t = [t for t, d in zip(t_out, dm) if d <= 1e-4]
    out = {"t": list(t_out), "max_dm_replayed": dm,
           "max_dm_control_fp64_strength_1e-9_replayed": md(c, a, t_out),
           "replay_forced_accepts": rb["replay"]["forced_accepts"], "plain_steps_recorded": int(len(steps[0])),
           "t_floor": list(t_floor), "max_dm_fp64_rtol1e-6_vs_rtol1e-8": md(f6, f8, t_floor),
           "bound": 1e-4, "holds_at_t": ok_t, "holds_everywhere": len(ok_t) == len(t_out)}
    if "learned_status" in rb:
        out["learned_status_in_replay"] = rb["learned_status"]
    return out


def e2e_run(args, form, world, rank):
    """Same metric through the public API from host buffers: pinned y0 and
    mask uploaded inside the timed region, one y(t) frame read back per step.
    The frames are read back on a copy stream from two alternating device
    buffers, so each device-to-host copy overlaps the next step's work (a
    buffer is written again only after its copy has finished)."""
    import torch
    p, g, o = form_params(form, 12345 + rank)
    n = p.ng * p.ny
    sub = max(1, int(round(args.dt / 0.1)))
    ctx2 = llg.Context(p)
    if FORMS[form]["learned"]:
        ctx2.learned_set_weights(train_weights(rank)[0])
    geo2 = llg.build_geometry(g, want=("active", "y0"))
    mask_h = torch.from_numpy(np.tile(geo2["active"].astype(np.float64), 3)).pin_memory()
    y0_h = torch.from_numpy(geo2["y0"]).pin_memory()
    frame_h = [torch.empty(3 * n, dtype=torch.float64).pin_memory() for _ in range(2)]
    y0_d = torch.empty(3 * n, dtype=torch.float64, device="cuda")
    yo_d = [torch.empty_like(y0_d) for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    copied = [None, None]
    torch.cuda.synchronize()
    dist_barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    ctx2.set_mask(mask_h.numpy())
    y0_d.copy_(y0_h, non_blocking=True)
    ctx2.integrator_init(0.0, y0_d, o)
    tt = 0.0
    main = torch.cuda.current_stream()
    for i in range(args.steps):
        b = i % 2
        if copied[b] is not None:
            main.wait_event(copied[b])   # the frame copy out of this buffer is done
        for k in range(sub):
            ctx2.integrate(tt + args.dt * (k + 1) / sub, yo_d[b])
        tt += args.dt
        done = torch.cuda.Event()
        done.record(main)
        copy_stream.wait_event(done)
        with torch.cuda.stream(copy_stream):
            frame_h[b].copy_(yo_d[b], non_blocking=True)
            copied[b] = torch.cuda.Event()
            copied[b].record(copy_stream)
    main.wait_stream(copy_stream)
    f1.record()
    torch.cuda.synchronize()
    ems = dist_max(f0.elapsed_time(f1), world)
    ctx2.close()
    return {"value": world * args.steps * args.dt / (ems / 1000.0), "unit": UNIT,
            "h2d_bytes_per_step": int((y0_h.numel() * 8 + mask_h.numel() * 8) / args.steps),
            "d2h_bytes_per_step": int(frame_h[0].numel() * 8),
            "note": "the timed window through the public API from host buffers: fresh instance from t=0, pinned "
                    "y0 + mask uploaded and the integrator set up inside the timed region (amortised over the "
                    "steps), one y(t) frame copied back per step on a copy stream, overlapping the next step"}


def run_ours(args, world, rank, local):
    import torch
    torch.cuda.set_device(local)
    lib = llg.load()
    form = args.form or BEST_FORM
    ng, ny = 1536, 512
    main = timed_run(args, form, world, rank, local, lib)
    roof = roofline_for(lib, main, ng, ny, FORMS[form]["demag_precision"] == llg.DEMAG_MIXED,
                        FORMS[form].get("krylov", llg.KRYLOV_FP64) == llg.KRYLOV_FP32)
    clk = main["clocks"].summary()
    main["ctx"].close()
    summary = {"form_ran": main["ran"], "value": main["value"]}
    compare = None
    if form != "plain" and not args.no_compare:
        plain = timed_run(args, "plain", world, rank, local, lib, clocks=False)
        plain["ctx"].close()
        compare = {"plain_fp64_value": plain["value"], "plain_fp64_ms_per_step": plain["ms"] / args.steps,
                   "ratio_vs_plain_fp64": main["value"] / plain["value"],
                   "gmres_iters_per_newton": main["counters"]["nli"] / max(main["counters"]["nni"], 1),
                   "plain_gmres_iters_per_newton": plain["counters"]["nli"] / max(plain["counters"]["nni"], 1),
                   "bdf_steps": main["counters"]["nst"], "plain_bdf_steps": plain["counters"]["nst"],
                   "plain_counters": plain["counters"]}
        for other in ("mixed", "mixed32", "learned+mixed", "learned+mixed32"):
            if other == form:
                continue
            r_ = timed_run(args, other, world, rank, local, lib, clocks=False)
            r_["ctx"].close()
            compare[f"{other}_value"] = r_["value"]
            compare[f"{other}_gmres_iters_per_newton"] = r_["counters"]["nli"] / max(r_["counters"]["nni"], 1)
            compare[f"{other}_bdf_steps"] = r_["counters"]["nst"]
        if not args.no_reference_gs:
            mgs = timed_run(args, "plain", world, rank, local, lib, clocks=False, gs=llg.GS_AUTO)
            mgs["ctx"].close()
            compare["plain_fp64_reference_gs_value"] = mgs["value"]
            compare["plain_fp64_reference_gs_note"] = ("plain FP64 with the reference's Gram-Schmidt choice at this "
                                                       "size (modified, neq >= 5e5)")
        summary.update(plain_fp64_value=plain["value"], ratio_vs_plain_fp64=compare["ratio_vs_plain_fp64"])
    accuracy = None
    if form != "plain" and not args.no_accuracy:
        try:
            accuracy = replay_accuracy(form, rank)
            ts = [str(t) for t in accuracy["t"]]
            summary.update(max_dm_replayed=dict(zip(ts, accuracy["max_dm_replayed"])),
                           max_dm_control_fp64_strength_1e9_replayed=dict(
                               zip(ts, accuracy["max_dm_control_fp64_strength_1e-9_replayed"])),
                           max_dm_fp64_rtol1e6_vs_rtol1e8=dict(zip([str(t) for t in accuracy["t_floor"]],
                                                                   accuracy["max_dm_fp64_rtol1e-6_vs_rtol1e-8"])),
                           accuracy_bound=1e-4, accuracy_holds_at_t=accuracy["holds_at_t"])
        except llg.LLGError as e:   # reported, not hidden: the line says the check did not complete
            accuracy = {"error": str(e)}
            summary.update(accuracy_error=str(e))
    e2e = None if args.no_e2e else e2e_run(args, form, world, rank)
    if e2e:
        summary["e2e_value"] = e2e["value"]
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args)
    line = {
        "metric": METRIC, "value": main["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": main["ms"] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded geometry/IC builders)",
        "config": bench_config(args, world),
        "form": FORMS[form]["desc"],
        "roofline": roof,
        "e2e": e2e, "gpu_launches": sum(main["launches"].values()), "clocks": clk, "cpu_baseline": cpu,
        "launches_by_family": main["launches"], "solver_counters_timed": main["counters"],
        "training": _weights_cache.get("info") if FORMS[form]["learned"] else None,
        "compare": compare, "accuracy": accuracy,
        "summary": summary,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_config4(args, world, rank, local):
    """The batched mixed workload: 64 independent instances of uneven size
    (256x256 .. 1024x512; square hole, annulus, compact ellipse, windowed
    polycrystal; open demag U[1,4]).  Every rank builds the same seeded list
    and integrates its longest-processing-time share (shard.py; no collective
    in the hot path), each instance on its own stream.  A step advances every
    instance by --dt.  value = instance sim-time of all 64 instances per
    wall-second (max over ranks: the whole job, fixed total work).  After the
    run one host gather brings every instance's final-state norm and step
    count to rank 0.  At N = 1 the same instances then continue one at a time
    (one host thread) for the sequential comparison."""
    import torch

    import shard
    torch.cuda.set_device(local)
    insts = llg.config4_instances(64, 12345)
    mine = shard.my_instances(insts, world, rank)
    part, load = shard.partition_lpt([shard.instance_cost(x["params"]) for x in insts], world)
    # classical Gram-Schmidt for every instance: the single-graph form runs the
    # device-resident step loop, which covers it (the reference would pick
    # modified Gram-Schmidt for the 1024x512 instances, neq >= 5e5)
    opts = llg.default_solver_opts(gs_type=llg.GS_CLASSICAL)
    t0 = time.perf_counter()
    b = llg.Batch([insts[i]["params"] for i in mine])
    y0 = [torch.from_numpy(llg.setup_instance(b.ctx[k], insts[i])).cuda() for k, i in enumerate(mine)]
    outs = [torch.zeros_like(y) for y in y0]
    b.integrator_init(0.0, y0, opts)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    t = 0.0

    def run(k, nthreads, graph=False):
        nonlocal t
        torch.cuda.synchronize()
        dist_barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(k):
            t += args.dt
            if graph:
                b.integrate_graph(t, outs)
            else:
                b.integrate(t, outs, nthreads=nthreads)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # warm-up: W output intervals of 0.1 (every instance; the first one is the
    # host start-up, the next ones build and run the single graph)
    for k in range(args.warmup):
        t += 0.1
        if k == 0:
            b.integrate(t, outs, nthreads=0)
        else:
            b.integrate_graph(t, outs)
    torch.cuda.synchronize()
    st0 = [s_["nst"] for s_ in b.stats()]
    with Clocks(local) as clk:
        ms_local = run(args.steps, 0, graph=True)
    ms = dist_max(ms_local, world)
    st1 = [s_["nst"] for s_ in b.stats()]
    ms_pool = dist_max(run(args.steps, 0), world)
    local_res = {i: {"rank": rank, "nst": int(st1[k]), "nst_timed": int(st1[k] - st0[k]),
                     "m_norm": float(torch.linalg.vector_norm(outs[k]).item())} for k, i in enumerate(mine)}
    merged = shard.gather_results(local_res, world, rank)
    seq = None
    if world == 1:
        ms_seq = run(args.steps, 1)
        seq = {"ms_per_step": ms_seq / args.steps, "value": len(insts) * args.steps * args.dt / (ms_seq / 1000.0),
               "speedup_concurrent": ms_seq / ms}
    cells = sum(x["params"].ng * x["params"].ny for x in insts)
    value = len(insts) * args.steps * args.dt / (ms / 1000.0)
    line = {
        "metric": "instance-sim-time/wall-s @64-instance mixed batch", "value": value,
        "unit": "instance-sim-time/wall-s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded config-4 generator, master seed 12345)",
        "config": {"workload": "64 instances: sizes {256x256,512x256,512x512,1024x512}, shapes {square hole, "
                               "annulus 0.15-0.35 N, ellipse 0.3x0.2 (compact), polycrystal 24 grains 10% dead "
                               "(windowed)}, open demag U[1,4], rtol 1e-4", "instances": len(insts),
                   "cells_total": cells, "sim_time_per_step": args.dt,
                   "form": "mixed-precision demag, block-Jacobi, classical Gram-Schmidt",
                   "launch": "every instance's device-resident step loop as one branch of ONE CUDA graph; one graph "
                             "launch per step advances all instances",
                   "parallelism": f"LPT split of the instances over {world} GPU(s)",
                   "setup_s": setup_s},
        "split": {"instances_per_rank": [int((part == r).sum()) for r in range(world)],
                  "cost_per_rank": [float(x) for x in load]},
        "host_driven_thread_pool": {"ms_per_step": ms_pool / args.steps,
                                    "value": len(insts) * args.steps * args.dt / (ms_pool / 1000.0),
                                    "note": "the same instances driven from a host thread pool, one stream each"},
        "sequential_same_instances": seq,
        "clocks": clk.summary(),
    }
    if rank == 0:
        line["bdf_steps_timed"] = int(sum(v["nst_timed"] for v in merged.values()))
        line["gathered_instances"] = len(merged)
    b.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def harvest_train(ctx, y0, o, t_end, w_init=None, seed=5):
    """Harvest block-Jacobi SPGMR solves of one instance over [0, t_end] and
    train on them (continuing from w_init when given)."""
    import torch
    if w_init is not None:
        ctx.learned_set_weights(w_init)
    ctx.learned_harvest(TRAIN["max_samples"], TRAIN["stride"])
    ctx.integrator_init(0.0, y0, o)
    yout = torch.zeros_like(y0)
    for k in range(1, int(round(t_end / 0.1)) + 1):
        ctx.integrate(0.1 * k, yout)
    l0, l1 = ctx.learned_train(iters=TRAIN["iters"], batch=TRAIN["batch"], patch=TRAIN["patch"], seed=seed,
                               lr=TRAIN["lr"], init_scale=TRAIN["init_scale"])
    return ctx.learned_get_weights(), {"samples": ctx.learned_num_samples(), "loss_first": l0, "loss_last": l1}


def run_config3(args, world, rank, local):
    """The compact-circle workload with the learned preconditioner: 2048x2048
    cells, EXEC_COMPACT active-index lists of the centred circle r = 0.25 N
    (19.6 % active), periodic FFT demag of strength 2 (the reference's
    un-padded convention), vortex state (-y, x, 0.1)/norm + 0.01 jitter,
    mixed-precision demag, rtol 1e-4, SPGMR(5).  The network is trained on
    solves harvested from the square-hole film (1536x512, open demag 4) and
    then the 72-grain polycrystal (1536x512, windowed demag 1); the circle is
    then integrated over t 0 -> --steps * --dt with block-Jacobi, with the
    learned preconditioner on every solve, and with the cost-aware policy.
    Reported: GMRES iterations per Newton iteration and sim-time/s of each."""
    import torch
    torch.cuda.set_device(local)
    lib = llg.load()
    t0 = time.perf_counter()
    # training on the two 1536x512 workloads
    p1, g1, o1 = workload(seed=12345 + rank)
    p1.demag_precision = llg.DEMAG_MIXED
    c1, geo1 = make_ctx(p1, g1)
    w, info1 = harvest_train(c1, torch.from_numpy(geo1["y0"]).cuda(), o1, 1.0)
    c1.close()
    p2 = llg.default_params(1536, 512, demag_mode=llg.DEMAG_OPEN, demag_strength=1.0, windowed=1, chb=0.0,
                            norm_kind=llg.NORM_REG, demag_precision=llg.DEMAG_MIXED, bc=llg.BC_FREE)
    g2 = llg.default_geom(1536, 512, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=72, dead_grain_frac=0.16,
                          grain_z_bias=1.0, ic_kind=llg.IC_TWO_DOMAIN_X, ic_jitter_eps=0.01, init_random_seed=12345)
    geo2 = llg.build_geometry(g2)
    c2 = llg.Context(p2)
    c2.set_window(geo2["w"], geo2["msk3"], geo2["nsk3"])
    w, info2 = harvest_train(c2, torch.from_numpy(geo2["y0"]).cuda(), o1, 0.5, w_init=w, seed=6)
    c2.close()
    train_s = time.perf_counter() - t0
    n = 2048
    g3 = llg.default_geom(n, n, geometry_kind=llg.GEOM_ELLIPSE, active_rx_frac=0.25, active_ry_frac=0.25,
                          ic_kind=llg.IC_VORTEX, ic_jitter_eps=0.01, init_random_seed=12345 + rank)
    geo3 = llg.build_geometry(g3)
    ids = np.arange(n * n, dtype=np.int32)
    act = geo3["active"]
    res = {}
    for name, kind, policy in (("block_jacobi", llg.PREC_BLOCK_JACOBI, None), ("learned_every_solve", llg.PREC_LEARNED, 0),
                               ("learned_cost_aware", llg.PREC_LEARNED, 1)):
        p3 = llg.default_params(n, n, exec_model=llg.EXEC_COMPACT, bc=llg.BC_PERIODIC, demag_mode=llg.DEMAG_PERIODIC,
                                demag_strength=2.0, norm_kind=llg.NORM_REG, demag_precision=llg.DEMAG_MIXED,
                                precond_kind=kind)
        ctx = llg.Context(p3)
        ctx.set_active_ids(ids[act == 1], ids[act == 0])
        if kind == llg.PREC_LEARNED:
            ctx.learned_set_weights(w)
            ctx.learned_set_policy(bool(policy))
        y0 = torch.from_numpy(geo3["y0"]).cuda()
        ctx.integrator_init(0.0, y0, llg.default_solver_opts())
        yout = torch.zeros_like(y0)
        for k in range(1, args.warmup + 1):   # warm-up output intervals (0.1 each)
            ctx.integrate(0.1 * k, yout)
        torch.cuda.synchronize()
        st0 = ctx.stats()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        tstart = 0.1 * args.warmup
        sub = max(1, int(round(args.dt / 0.1)))
        e0.record()
        for s_ in range(args.steps):
            for k in range(sub):
                ctx.integrate(tstart + s_ * args.dt + args.dt * (k + 1) / sub, yout)
        e1.record()
        torch.cuda.synchronize()
        st1 = ctx.stats()
        ms = e0.elapsed_time(e1)
        d = {k: st1[k] - st0[k] for k in ("nst", "nni", "nli", "nfe")}
        res[name] = {"gmres_iters_per_newton": d["nli"] / max(d["nni"], 1), "sim_time_per_s":
                     args.steps * args.dt / (ms / 1000.0), "counters": d}
        if kind == llg.PREC_LEARNED:
            res[name]["learned_status"] = ctx.learned_status()
        ctx.close()
    line = {
        "metric": "GMRES iterations per Newton iteration @2048x2048 compact circle, learned vs block-Jacobi",
        "value": res["learned_every_solve"]["gmres_iters_per_newton"], "unit": "iterations/Newton",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
        "dtype": "f64", "data": "synthetic (seeded builders)",
        "config": {"workload": "2048x2048 cells, EXEC_COMPACT circle r=0.25 N (19.6 % active), periodic FFT demag "
                               "strength 2, vortex (-y,x,0.1)/norm + 0.01 jitter, mixed-precision demag, rtol 1e-4, "
                               "SPGMR(5)", "window": f"t {0.1 * args.warmup:g} -> "
                                                     f"{0.1 * args.warmup + args.steps * args.dt:g}",
                   "n_active": int(act.sum())},
        "block_jacobi": res["block_jacobi"], "learned_every_solve": res["learned_every_solve"],
        "learned_cost_aware": res["learned_cost_aware"],
        "training": {"square_hole_1536x512": info1, "polycrystal_1536x512": info2, "train_s": train_s},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_config2(args, world, rank, local):
    """The polycrystal workload with the mixed-precision form: 1536x512 cells,
    72 Voronoi grains from seeded sites, 16 % dead, axes uniform on the sphere,
    windowed open demag of strength 1, two domains (+x left, -x right) with
    0.01 jitter, rtol 1e-4.  Each form is timed over t 0 -> steps*dt from a
    fresh instance; then the mixed forms replay plain FP64's recorded steps
    over the same window and max|dm| against FP64 is reported at t = 1, 5
    and the end, beside an FP64 control whose demag strength is changed by
    1e-9 (same steps), which measures how much the film itself amplifies a
    perturbation."""
    import torch
    torch.cuda.set_device(local)
    n_ng, n_ny = 1536, 512
    g = llg.default_geom(n_ng, n_ny, geometry_kind=llg.GEOM_POLYCRYSTAL, num_grains=72, dead_grain_frac=0.16,
                         grain_z_bias=1.0, ic_kind=llg.IC_TWO_DOMAIN_X, ic_jitter_eps=0.01,
                         init_random_seed=12345 + rank)
    geo = llg.build_geometry(g)
    t_end = args.steps * args.dt
    kmax = int(round(t_end / 0.1))

    t_marks = [t for t in (1.0, 5.0) if t < t_end] + [t_end]
    k_marks = {int(round(t / 0.1)): t for t in t_marks}

    def run(prec, krylov, record=False, replay=None, timed=False, strength=1.0):
        p = llg.default_params(n_ng, n_ny, demag_mode=llg.DEMAG_OPEN, demag_strength=strength, windowed=1,
                               norm_kind=llg.NORM_REG, bc=llg.BC_FREE, demag_precision=prec)
        ctx = llg.Context(p)
        ctx.set_window(geo["w"], geo["msk3"], geo["nsk3"])
        y0 = torch.from_numpy(geo["y0"]).cuda()
        ctx.integrator_init(0.0, y0, llg.default_solver_opts(gs_type=GS, krylov_precision=krylov))
        if record:
            ctx.record_steps(10_000_000)
        if replay is not None:
            ctx.replay_steps(*replay)
        yout = torch.zeros_like(y0)
        marks = {}
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(1, kmax + 1):
            ctx.integrate(0.1 * k, yout)
            if not timed and k in k_marks:
                marks[k_marks[k]] = yout.cpu().numpy()   # (accuracy runs only: the copy is not timed)
        e1.record()
        torch.cuda.synchronize()
        out = {"y": yout.cpu().numpy(), "ms": e0.elapsed_time(e1), "stats": ctx.stats(), "marks": marks}
        if record:
            out["steps"] = ctx.recorded_steps()
        ctx.close()
        return out

    run(llg.DEMAG_MIXED, llg.KRYLOV_FP64)    # warm-up (module load, autotune of this transform size)
    res = {}
    for name, prec, kr in (("plain", llg.DEMAG_FP64, llg.KRYLOV_FP64), ("mixed", llg.DEMAG_MIXED, llg.KRYLOV_FP64),
                           ("mixed32", llg.DEMAG_MIXED, llg.KRYLOV_FP32)):
        r_ = run(prec, kr, record=(name == "plain"), timed=True)
        res[name] = r_
    # accuracy: FP64 recorded again with its marks (the timed runs copy nothing out)
    ref = run(llg.DEMAG_FP64, llg.KRYLOV_FP64, replay=res["plain"]["steps"])
    acc = {}
    for name, prec, kr, st in (("mixed", llg.DEMAG_MIXED, llg.KRYLOV_FP64, 1.0),
                               ("mixed32", llg.DEMAG_MIXED, llg.KRYLOV_FP32, 1.0),
                               ("control_fp64_strength_1e-9", llg.DEMAG_FP64, llg.KRYLOV_FP64, 1.0 + 1e-9)):
        r_ = run(prec, kr, replay=res["plain"]["steps"], strength=st)
        acc[name] = {str(t): float(np.abs(r_["marks"][t] - ref["marks"][t]).max()) for t in t_marks}
    val = {k: t_end / (v["ms"] / 1000.0) for k, v in res.items()}
    line = {
        "metric": "sim-time/wall-s @1536x512 polycrystal, mixed vs plain FP64", "value": val["mixed32"],
        "unit": "sim-time/wall-s", "n_gpus": world, "steps": args.steps, "warmup": 1, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic (seeded builders)",
        "config": {"workload": "1536x512 cells, 72 Voronoi grains (16 % dead, axes uniform), windowed open demag "
                               "strength 1, two domains +-x with 0.01 jitter, rtol 1e-4, SPGMR(5), block-Jacobi",
                   "window": f"fresh instance, t 0 -> {t_end:g}"},
        "values": val, "bdf_steps": {k: v["stats"]["nst"] for k, v in res.items()},
        "gmres_iters_per_newton": {k: v["stats"]["nli"] / max(v["stats"]["nni"], 1) for k, v in res.items()},
        "max_dm_vs_plain_fp64_replayed": acc,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def cpu_oracle_run(dt_step, steps, warmup_intervals, threads):
    """The oracle (C, OpenMP) on the bench workload: warm-up output intervals
    of 0.1 on a throwaway instance, then `steps` steps of dt_step from t = 0
    on a fresh instance, each at the 0.1 output cadence."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import binding
    binding.build()
    used = binding.set_threads(threads)
    p, g, o = workload()
    geo = binding.build_geometry(g)

    def instance():
        orc = binding.Oracle(p)
        orc.set_active(geo["active"])
        orc.integrator_init(geo["y0"], o)
        return orc

    def advance(orc, t0, t1):
        k0, k1 = int(round(t0 / 0.1)), int(round(t1 / 0.1))
        for k in range(k0 + 1, k1 + 1):
            rc, _, _ = orc.integrate(0.1 * k)
            if rc != 0:
                raise RuntimeError(f"oracle integrate rc={rc}")
        if abs(t1 - 0.1 * k1) > 1e-12:
            rc, _, _ = orc.integrate(t1)
            if rc != 0:
                raise RuntimeError(f"oracle integrate rc={rc}")

    w = instance()
    advance(w, 0.0, 0.1 * warmup_intervals)
    del w
    orc = instance()
    t = 0.0
    t0 = time.perf_counter()
    for _ in range(steps):
        advance(orc, t, t + dt_step)
        t += dt_step
    el = time.perf_counter() - t0
    return steps * dt_step / el, used, el, orc.stats()


def cpu_baseline(args):
    threads = os.cpu_count() or 1
    val, used, el, st = cpu_oracle_run(args.cpu_dt, args.cpu_steps, 1, threads)
    return {"value": val, "unit": UNIT, "cores": used, "kind": "port",
            "sample": f"same 1536x512+open-demag workload, fresh instance, {args.cpu_steps} steps of {args.cpu_dt} "
                      f"sim-time from t=0 ({el:.1f} s CPU wall, {st['nst']} BDF steps); C FP64 restatement of the "
                      "reference path with OpenMP (the full window runs under --impl reference)",
            "cpu_model": cpu_model()}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return None


def run_reference(args, world, rank):
    """The reference arm: the CPU restatement of the reference path over the
    same window as the GPU arm (fresh instance, t 0 -> K*dt), all host cores."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    val, used, el, st = cpu_oracle_run(args.dt, args.steps, args.warmup, threads)
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1000.0 * el / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded geometry/IC builders)",
        "config": bench_config(args, world),
        "form": "plain FP64 (CPU restatement of the reference path: same RHS, demag, Jv, block-Jacobi, "
                "CVODE-equivalent BDF/Newton/SPGMR with classical Gram-Schmidt)",
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": used, "kind": "port",
                         "sample": f"the full window: {args.steps} steps of {args.dt} sim-time from t=0 on a fresh "
                                   f"instance ({st['nst']} BDF steps, {el:.1f} s); CPU FP64 restatement of the "
                                   "reference path (SUNDIALS absent, so the reference solver itself cannot be "
                                   "built)", "cpu_model": cpu_model()},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "solver_counters": {k: st[k] for k in ("nst", "nfe", "nni", "nli", "nsetups", "netf", "ncfn")},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--dt", type=float, default=1.0)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-dt", type=float, default=0.1)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-accuracy", action="store_true", help="skip the replayed accuracy runs")
    ap.add_argument("--no-reference-gs", action="store_true",
                    help="skip the plain FP64 run with the reference's Gram-Schmidt choice")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--form", choices=sorted(FORMS), default=None,
                    help="form to time (default: the best one built, compared against plain FP64)")
    ap.add_argument("--no-compare", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--profile-window", action="store_true",
                    help="cudaProfilerStart/Stop around the timed steps (ncu --profile-from-start off)")
    ap.add_argument("--workload", choices=["1536x512", "config2", "config3", "config4"], default="1536x512",
                    help="config3: the compact circle with the learned preconditioner; config4: the 64-instance "
                         "batched workload (each its own JSON line)")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload == "config4":
            run_config4(args, world, rank, local)
        elif args.workload == "config3":
            run_config3(args, world, rank, local)
        elif args.workload == "config2":
            run_config2(args, world, rank, local)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
