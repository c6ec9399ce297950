"""Benchmark of WAM Cycle 7's per-time-step hot path on B200.

Metric: spectral-point updates per second (one bin = one (sea point,
direction, frequency) advanced by one source step IDELT together with its
IDELT/IDELPRO propagation steps), forward, FP32.

Workload (default): the 0.1-degree regional configuration, 1200x900 grid
(45S-45N, 60W-60E) with ~30% seeded blob land (~760k sea points), depth
10-5000 m from a seeded Gaussian random field, KL=36 x ML=30 spectrum
(FR1=0.0345 Hz), ST6 physics (IPHYS=2), spherical shallow-water propagation
with depth refraction, IDELPRO=120 s, IDELT=600 s.  One step = 5 PROPAGS +
1 IMPLSCH.  Inputs are seeded synthetic fields (no dataset exists for this
path); the spectrum (3.3 GB) is far larger than L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl wamgpu|reference]

--impl reference times the CPU restatement of the reference (oracle/, the
reference's Fortran cannot be compiled on these machines) with all host
threads on latitude bands of the same workload grid (same config line).  With N>1 (torchrun), every
rank runs its own replica of the workload (weak scaling, no collective).
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "spectral-pt updates/s fwd, adjoint, batched on 1 B200 at Hs rel err<=1e-4"
UNIT = "spectral-point updates/s"
FALLBACK_HBM = 6650.0  # GB/s, used only if MEASURED_PEAKS.json is absent


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="wamgpu", choices=["wamgpu", "reference"])
    p.add_argument("--workload", default="c1")
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-batched", action="store_true")
    p.add_argument("--no-adjoint", action="store_true")
    p.add_argument("--only", choices=["batched", "adjoint", "adjoint_st6"], default=None,
                   help="run only the batched-ensemble or the adjoint-window section and print its object "
                        "(for profiling those kernels; not a bench line)")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # nominal: SMs x FP32 lanes x 2 (FMA) x max SM clock


def fp32_roofline(workload, kernels, bins):
    """FP32 roofline of IMPLSCH: the algorithm's floating-point operations per
    bin (the oracle run with a counting number type, profiles/op_counts.json
    written by oracle/count_ops.py) times the bins of one launch, over the
    launch's CUDA-event time, against the nominal FP32 peak."""
    path = os.path.join(ROOT, "profiles", "op_counts.json")
    key = f"implsch_{workload}"
    if "implsch" not in kernels or not os.path.exists(path):
        return None
    with open(path) as f:
        ops = json.load(f)
    if key not in ops:
        return None
    fpb = ops[key]["flops_per_bin"]
    ach = fpb * bins / (kernels["implsch"]["avg_ms"] / 1e3) / 1e12
    return {"kernel": "implsch", "achieved": ach, "peak": FP32_PEAK_TFLOPS, "unit": "TFLOP/s",
            "frac": ach / FP32_PEAK_TFLOPS, "flops_per_bin": fpb,
            "transcendentals_per_bin": ops[key]["per_bin"]["trans"],
            "peak_kind": "nominal (148 SMs x 128 FP32 lanes x 2 x 1965 MHz)",
            "counts": "profiles/op_counts.json (oracle/count_ops.py)"}


def workload_config(name, scale, nsea, kl, ml):
    """The `config` of both arms: the workload, its sea points and bins per point."""
    if name == "c1" and scale == 1.0:
        desc = ("c1: 0.1 deg 1200x900 regional, ST6, KL=36 ML=30, IDELPRO=120 s IDELT=600 s "
                "(5 PROPAGS + 1 IMPLSCH per step)")
    else:
        desc = f"{name} at scale {scale}"
    return {"workload": desc, "nsea": int(nsea), "bins_per_point": int(kl * ml)}


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


class CpuSample:
    """The oracle (the CPU restatement of the reference) on bands of the
    full workload grid: each band is a contiguous range of the south-to-north
    ordered sea points with the halo rows its propagation reads, prepared once
    (PREPARE_PROPAGATION with its stored coefficient arrays, as the reference
    does) and kept resident in the oracle's REAL precision.  One CPU step runs
    one band's WAMODEL pass (IDELT/IDELPRO PROPAGS calls, then IMPLSCH over
    every point of the band) on all host threads; the bands take turns.  The
    bins counted are all the points the pass updates, halo rows included."""

    def __init__(self, name, scale, nbands=64, sample_bands=(8, 24, 40, 56)):
        from oracle.oracle import Oracle
        from wam_b200.halo import local_grid, partition
        from wam_b200.synth import make_workload
        w = make_workload(name, scale=scale)
        self.w = w
        self.nprop = w.cfg["idelt"] // w.cfg["idelpro"]
        self.nthreads = os.cpu_count() or 1
        parts = partition(w.grid, nbands)
        self.bands = []
        f_all = None
        for q in sample_bands:
            p = parts[min(q, nbands - 1)]
            a, b = p["ninf"], p["nsup"]
            o = Oracle(w.cfg)
            o.set_grid(local_grid(w.grid, p))
            o.set_fields(w.depth[a:b])
            o.prepare_propagation()
            o.prepare_source()
            e = w.e_fm[a:b]
            d = w.d_fk[a:b]
            f = np.asfortranarray(e[:, None, :] * d[:, :, None])
            sl = lambda x: np.asarray(x)[a:b]
            o.resident_set(f, sl(w.u10), sl(w.udir), sl(w.tauw), sl(w.ustar), sl(w.z0), sl(w.roairn), sl(w.wstar),
                           sl(w.depth))
            self.bands.append((o, b - a))
        self.i = 0

    def step(self):
        """One band's pass; returns (bins updated, seconds)."""
        o, n = self.bands[self.i % len(self.bands)]
        self.i += 1
        t0 = time.perf_counter()
        o.resident_step(self.nprop, self.nthreads)
        dt = time.perf_counter() - t0
        return n * self.w.cfg["kl"] * self.w.cfg["ml"], dt

    def describe(self, nsteps, seconds):
        pts = [n for _, n in self.bands]
        return (f"{len(pts)} latitude bands of the full {self.w.grid['nx']}x{self.w.grid['ny']} grid "
                f"({min(pts)}-{max(pts)} sea points each, halo rows included) taking turns, {nsteps} WAMODEL "
                f"passes ({self.nprop} PROPAGS + IMPLSCH) in {seconds:.1f} s on {self.nthreads} host threads "
                f"({cpu_model()})")


def cpu_baseline(name, scale, budget_s):
    """cpu_baseline object of the GPU arm: the oracle sample for ~budget_s seconds."""
    cs = CpuSample(name, scale)
    cs.step()  # warm
    bins = secs = 0.0
    n = 0
    while secs < budget_s:
        b, dt = cs.step()
        bins += b
        secs += dt
        n += 1
    return {"value": bins / secs, "unit": UNIT, "cores": cs.nthreads, "kind": "port", "cpu": cpu_model(),
            "sample": cs.describe(n, secs)}


def run_reference(args):
    """The reference arm: the CPU restatement of the reference's path (the
    Fortran reference cannot be built on these machines) timed on the host
    cores on bands of the same workload grid, same config and metric as the
    GPU arm.  Rank 0 alone runs it under torchrun."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cs = CpuSample(args.workload, args.scale)
    for _ in range(args.warmup):
        cs.step()
    bins = secs = 0.0
    for _ in range(args.steps):
        b, dt = cs.step()
        bins += b
        secs += dt
    val = bins / secs
    w = cs.w
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded fields; no dataset for this path)",
            "config": workload_config(args.workload, args.scale, w.nsea, w.cfg["kl"], w.cfg["ml"]),
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": cs.nthreads, "kind": "port", "cpu": cpu_model(),
                             "sample": cs.describe(args.steps, secs)},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def transfer_bound(torch, dev, hf, reps=3):
    """The host link for the e2e step's bytes: the pinned spectrum copied up
    alone, down alone, and both at once on two streams (best of `reps`, wall
    clock around synchronised copies).  The e2e step cannot beat the
    concurrent figure."""
    up_dst = torch.empty(hf.numel(), dtype=hf.dtype, device=dev)
    down_src = torch.empty_like(up_dst)
    down_dst = torch.empty(hf.numel(), dtype=hf.dtype, pin_memory=True)
    src = hf.view(-1)
    su, sd = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def timed(up, down):
        best = None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            if up:
                with torch.cuda.stream(su):
                    up_dst.copy_(src, non_blocking=True)
            if down:
                with torch.cuda.stream(sd):
                    down_dst.copy_(down_src, non_blocking=True)
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
            best = t if best is None else min(best, t)
        return best

    nbytes = src.numel() * src.element_size()
    t_up, t_down, t_both = timed(True, False), timed(False, True), timed(True, True)
    return {"spectrum_bytes": nbytes, "h2d_gbs": nbytes / t_up / 1e9, "d2h_gbs": nbytes / t_down / 1e9,
            "both_directions_ms": 1e3 * t_both, "sequential_ms": 1e3 * (t_up + t_down)}


def batched_ensemble(dev, steps, warmup, n_members=32):
    """The 32-member ensemble (uneven regional grids, mixed KL/ML and ST4/ST6,
    900 s steps): one autotuned batched pass replayed from a CUDA graph per
    step, against the same members advanced one after another by their own
    wamgpu_step_dev on the same stream.  Device time by CUDA events."""
    import torch
    from wam_b200 import WamModel
    from wam_b200.batch import WamBatch
    from wam_b200.synth import make_ensemble
    ws = make_ensemble(n_members=n_members)
    models, states = [], []
    for w in ws:
        m = WamModel(dict(w.cfg, device=dev.index))
        m.set_grid(w.grid)
        m.set_depth(w.depth)
        m.prepare_propagation()
        m.prepare_source()
        models.append(m)
        t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
        f = w.spectrum_device(torch, dev)
        states.append([f, torch.empty_like(f)] + [t(a) for a in (w.u10, w.udir, w.tauw, w.ustar, w.z0, w.roairn,
                                                                  w.wstar)])
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream

    def sequential():
        for w, m, st in zip(ws, models, states):
            f, sc, u10, udir, tauw, ustar, z0, roairn, wstar = st
            m.step_dev(f, w.cfg["idelt"] // w.cfg["idelpro"], u10, udir, tauw, ustar, z0, roairn, wstar,
                       scratch=sc, stream=sh)

    def timed(fn):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    def sequential_synced():
        for w, m, st in zip(ws, models, states):
            f, sc, u10, udir, tauw, ustar, z0, roairn, wstar = st
            m.step_dev(f, w.cfg["idelt"] // w.cfg["idelpro"], u10, udir, tauw, ustar, z0, roairn, wstar,
                       scratch=sc, stream=sh)
            stream.synchronize()  # a plain run per member: its pass ends before the next member's starts

    ms_seq = timed(sequential)
    ms_seq_sync = timed(sequential_synced)
    b = WamBatch(models)
    for g, st in enumerate(states):
        b.set_member(g, *st)
    P, bs = b.tune(stream=sh)
    b.capture(stream=sh)
    ms_bat = timed(lambda: b.step(stream=sh))
    b.sync()
    bins = sum(w.nsea * w.cfg["kl"] * w.cfg["ml"] for w in ws)
    nbytes = sum(w.nsea * (8 * w.cfg["kl"] * w.cfg["ml"] + 48) * (1 + (w.cfg["idelt"] // w.cfg["idelpro"]) * m.counter)
                 for w, m in zip(ws, models))
    out = {"workload": f"c3: {n_members}-member ensemble, {sum(w.nsea for w in ws)} sea points in total "
                       f"({min(w.nsea for w in ws)}-{max(w.nsea for w in ws)} per member), KLxML 24x25/36x30, "
                       f"ST4/ST6 alternating, 900 s steps",
           "value": bins / (ms_bat / 1e3), "unit": UNIT, "ms_per_step": ms_bat,
           "sequential": {"value": bins / (ms_seq / 1e3), "ms_per_step": ms_seq,
                          "how": "each member's own wamgpu_step_dev, one after another on one stream, "
                                 "queued without waiting (the most favourable sequential form)"},
           "sequential_synchronised": {"value": bins / (ms_seq_sync / 1e3), "ms_per_step": ms_seq_sync,
                                       "how": "each member's own wamgpu_step_dev, the host waiting for each "
                                              "member's pass before the next, as 32 separate runs do"},
           "speedup_vs_sequential": ms_seq / ms_bat,
           "speedup_vs_sequential_synchronised": ms_seq_sync / ms_bat,
           "tuned": {"implsch_points_per_cta": P, "propags_points_per_cta": bs},
           "graph": True, "achieved_gbs": nbytes / (ms_bat / 1e3) / 1e9}
    b.close()
    for m in models:
        m.close()
    return out


def adjoint_window(dev, warmup, passes=24, n_obs=2000, seed=4242, scale=1.0, name="c2"):
    """Adjoint of one assimilation window on the 400x300 regional grid
    (KL=36, ML=30, ST4, IDELPRO=120 s, IDELT=600 s), FP32, through the C ABI
    an assimilation driver calls.  name="c1" with scale=1/3 is the same grid
    size on the ST6 regional recipe.

    The forward sweep runs `passes` WAMODEL passes with wamgpu_step_ckpt_dev,
    one checkpoint per pass (the spectrum entering IMPLSCH, TAUW, U10).  The
    cost is the squared Hs misfit at n_obs seeded sea points against a
    perturbed-truth run (U10 +10%) with Hs noise of sigma 0.2 m.  The backward
    sweep adds each pass's misfit adjoint at the observed points and runs
    wamgpu_step_adj_dev (the IMPLSCH adjoint from the checkpoint, then the
    PROPAGS transposes), giving the gradient with respect to the initial
    spectrum, the initial TAUW and each pass's U10.  Device times by CUDA
    events: the plain forward pass (wamgpu_step_dev), the checkpointed forward
    sweep and the backward sweep."""
    import torch
    from wam_b200 import WamModel
    from wam_b200.adjoint import significant_wave_height
    from wam_b200.synth import make_workload
    w = make_workload(name, scale=scale, device=dev.index)
    n_obs = min(n_obs, w.nsea)
    m = WamModel(w.cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    _, counter = m.prepare_propagation()
    m.prepare_source()
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    sh = stream.cuda_stream
    t = lambda a: torch.tensor(np.asarray(a, np.float32), device=dev)
    f0 = w.spectrum_device(torch, dev)
    u10, udir, tauw, roairn, wstar = (t(a) for a in (w.u10, w.udir, w.tauw, w.roairn, w.wstar))
    ustar, z0 = t(w.ustar), t(w.z0)
    nprop = w.cfg["idelt"] // w.cfg["idelpro"]
    u_seq = [u10 * (1.0 + 0.05 * (p // 6)) for p in range(passes)]  # hourly changes of the forcing
    gen = torch.Generator(device=dev).manual_seed(seed)
    points = torch.randperm(w.nsea, generator=gen, device=dev)[:n_obs]
    dfim = torch.tensor(m.table("DFIM"), device=dev, dtype=torch.float32)
    sc = torch.empty_like(f0)
    # perturbed truth and observations
    f, tw, obs = f0.clone(), tauw.clone(), []
    for u in u_seq:
        m.step_dev(f, nprop, 1.1 * u, udir, tw, ustar, z0, roairn, wstar, scratch=sc, stream=sh)
        hs = significant_wave_height(f, dfim, points)
        obs.append(hs + 0.2 * torch.randn(hs.shape, generator=gen, device=dev))
    ld = f0.shape[-1]
    m.checkpoint_reserve(passes, ld)
    ev = lambda: torch.cuda.Event(enable_timing=True)

    def plain():
        f, tw = f0.clone(), tauw.clone()
        torch.cuda.synchronize()
        e0, e1 = ev(), ev()
        e0.record(stream)
        for u in u_seq:
            m.step_dev(f, nprop, u, udir, tw, ustar, z0, roairn, wstar, scratch=sc, stream=sh)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / passes

    def window(np_):
        """One window of np_ passes: (cost, gradients, forward ms, backward ms)."""
        f, tw = f0.clone(), tauw.clone()
        lam_f, lam_t = torch.zeros_like(f0), torch.zeros_like(tauw)
        lam_u = [torch.empty_like(u10) for _ in range(np_)]
        torch.cuda.synchronize()
        e0, e1, e2 = ev(), ev(), ev()
        e0.record(stream)
        hs = []
        for p in range(np_):
            m.step_ckpt_dev(p, f, nprop, u_seq[p], udir, tw, ustar, z0, roairn, wstar, scratch=sc, stream=sh)
            hs.append(significant_wave_height(f, dfim, points))
        e1.record(stream)
        for p in reversed(range(np_)):
            # dJ/dF at the observed points: J = sum (Hs - obs)^2, Hs = 4 sqrt(E), E = sum DFIM sum F
            g = 16.0 * (hs[p] - obs[p]) / hs[p]
            lam_f[:, :, points] += dfim[:, None, None] * g[None, None, :]
            m.step_adj_dev(p, nprop, lam_f, lam_t, lam_u[p], udir, roairn, wstar, scratch=sc, stream=sh)
        e2.record(stream)
        torch.cuda.synchronize()
        J = sum(float(((h - o) ** 2).sum()) for h, o in zip(hs, obs))
        return J, lam_f, lam_t, lam_u, e0.elapsed_time(e1) / np_, e1.elapsed_time(e2) / np_

    for _ in range(warmup):
        plain()
    ms_plain = plain()
    window(2)  # warm-up
    J, lam_f, lam_t, lam_u, ms_fwd, ms_adj = window(passes)
    finite = bool(torch.isfinite(lam_f).all()) and all(bool(torch.isfinite(u).all()) for u in lam_u)
    bins = w.nsea * w.cfg["kl"] * w.cfg["ml"]
    if name == "c2":
        grid = "c2: 400x300 regional" if scale == 1.0 else f"c2: 400x300 regional recipe at scale {scale}"
    else:
        grid = f"{name} regional recipe at scale {scale:.4g}"
    phys = "ST4" if w.cfg["iphys"] == 1 else "ST6"
    out = {"workload": f"{grid}, {w.nsea} sea points, {phys}, KL=36 ML=30, IDELPRO=120 s IDELT=600 s, "
                       f"{passes}-pass window, {n_obs} Hs observations",
           "value": bins / (ms_adj / 1e3), "unit": UNIT + " (adjoint pass)", "ms_per_adjoint_pass": ms_adj,
           "ms_per_forward_pass": ms_plain, "ms_per_checkpointed_forward_pass": ms_fwd,
           "adjoint_over_forward": ms_adj / ms_plain, "counter": counter, "cost": J, "gradients_finite": finite,
           "checkpoint_bytes": passes * (bins + 3 * w.nsea) * 4,
           "how": "C ABI: forward = wamgpu_step_ckpt_dev per pass; backward = the misfit adjoint at the observed "
                  "points, then wamgpu_step_adj_dev per pass (IMPLSCH adjoint recomputing the source terms from "
                  "the checkpoint, then IDELT/IDELPRO PROPAGS transposes); plain forward = wamgpu_step_dev"}
    m.checkpoint_reserve(0, ld)
    m.close()
    torch.cuda.set_stream(torch.cuda.default_stream(dev))
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    import torch.distributed as dist
    from wam_b200 import WamModel
    from wam_b200.synth import make_workload

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if args.only:
        dev = torch.device("cuda", local)
        if args.only == "batched":
            out = batched_ensemble(dev, max(3, min(args.steps, 10)), max(3, args.warmup))
        elif args.only == "adjoint":
            out = adjoint_window(dev, max(3, args.warmup), scale=args.scale)
        else:
            out = adjoint_window(dev, max(3, args.warmup), passes=12, scale=args.scale / 3.0, name="c1")
        print(json.dumps({"section": args.only, **out}), flush=True)
        return
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    w = make_workload(args.workload, scale=args.scale, device=local)
    cfg = dict(w.cfg, device=local)
    m = WamModel(cfg)
    m.set_grid(w.grid)
    m.set_depth(w.depth)
    cfl, counter = m.prepare_propagation()
    m.prepare_source()
    n, KL, ML = w.nsea, cfg["kl"], cfg["ml"]
    nprop = cfg["idelt"] // cfg["idelpro"]
    ld = (n + 31) // 32 * 32
    F = w.spectrum_device(torch, dev, ld=ld)
    S = torch.empty_like(F)
    t = lambda a: torch.tensor(np.asarray(a), dtype=torch.float32, device=dev)
    u10, udir, roairn, wstar = t(w.u10), t(w.udir), t(w.roairn), t(w.wstar)
    tauw, ustar, z0 = t(w.tauw), t(w.ustar), t(w.z0)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream(dev)  # a non-default stream: handle 0 would select the library's own stream

    def step():
        m.step_dev(F, nprop, u10, udir, tauw, ustar, z0, roairn, wstar, scratch=S, ld=ld, stream=stream.cuda_stream)

    torch.cuda.set_stream(stream)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    m.timing()  # discard warm-up timings
    m.set_timing(True)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    kt = m.timing()
    m.set_timing(False)
    m.sync()
    ms_t = torch.tensor([ms], device=dev)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    bins = n * KL * ML
    value = world * bins * args.steps / (ms / 1e3)
    # roofline of the dominant kernel (algorithmic bytes: FL3 read + write + 12 per-point words)
    hbm, hbm_kind = peaks()
    per_launch_bytes = n * (8 * KL * ML + 48)
    kernels = {}
    for name, (kms, cnt) in kt.items():
        if cnt:
            avg = kms / cnt
            kernels[name] = {"launches": cnt, "avg_ms": avg, "share": kms / max(ms, 1e-9),
                             "achieved_gbs": per_launch_bytes / (avg / 1e3) / 1e9}
    dom = max(kernels, key=lambda k: kernels[k]["avg_ms"] * kernels[k]["launches"])
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(prof):
        with open(prof) as f:
            tr = json.load(f)
        key = f"{dom}_{args.workload}"
        if key in tr:
            traffic = tr[key]["dram_bytes_per_point"] * n
    roof = {"bound": "hbm", "achieved": kernels[dom]["achieved_gbs"], "peak": hbm, "unit": "GB/s",
            "frac": kernels[dom]["achieved_gbs"] / hbm, "traffic": traffic, "kernel": dom,
            "peak_kind": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback"}
    fp32 = fp32_roofline(args.workload, kernels, bins)
    if fp32:
        roof["fp32"] = fp32
    # end to end through the C ABI with host buffers (pinned): FL3 and the point fields in, results back
    e2e = None
    if not args.no_e2e and rank == 0:
        m2 = m
        hf = torch.empty((ML, KL, n), dtype=torch.float32, pin_memory=True)
        hf.copy_(F[:, :, :n])
        pin = lambda a: torch.tensor(np.asarray(a), dtype=torch.float32).pin_memory()
        hu, hd, hr, hw = pin(w.u10), pin(w.udir), pin(w.roairn), pin(w.wstar)
        ht, hs, hz = tauw.cpu().pin_memory(), ustar.cpu().pin_memory(), z0.cpu().pin_memory()
        fp = lambda x: x.numpy()
        arr = hf.numpy()
        fmt = np.lib.stride_tricks.as_strided(arr, shape=(n, KL, ML), strides=(4, 4 * n, 4 * n * KL))
        m2.step(fmt, nprop, fp(hu), fp(hd), fp(ht), fp(hs), fp(hz), fp(hr), fp(hw))  # warm
        ksteps = max(2, min(args.steps, 5))
        t0 = time.perf_counter()
        for _ in range(ksteps):
            m2.step(fmt, nprop, fp(hu), fp(hd), fp(ht), fp(hs), fp(hz), fp(hr), fp(hw))
        dt = time.perf_counter() - t0
        h2d = 4 * (n * KL * ML + 7 * n)
        d2h = 4 * (n * KL * ML + 3 * n)
        e2e = {"value": bins * ksteps / dt, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "steps": ksteps, "ms_per_step": 1e3 * dt / ksteps,
               "how": "wamgpu_step_host on pinned host FL3 + fields: H2D, 5 PROPAGS + IMPLSCH, D2H each step",
               "transfer_bound": transfer_bound(torch, dev, hf)}
    cpu = None
    if not args.no_cpu_baseline and rank == 0 and world == 1:
        cpu = cpu_baseline(args.workload, args.scale, 15.0)
    if rank == 0:
        launches = sum(v["launches"] for v in kernels.values())
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded fields; no dataset for this path)",
                "config": workload_config(args.workload, args.scale, n, KL, ML),
                "run": {"counter": counter, "total_cfl": cfl, "l2": "spectrum 3.3 GB >> 126 MB L2, no flush needed",
                        "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
                "roofline": roof, "kernels": kernels, "cpu_baseline": cpu, "e2e": e2e,
                "gpu_launches": launches, "clocks": clk.summary()}
        if not args.no_batched and world == 1:
            line["batched"] = batched_ensemble(dev, max(3, min(args.steps, 10)), max(3, args.warmup))
        if not args.no_adjoint and world == 1:
            line["adjoint"] = adjoint_window(dev, max(3, args.warmup))
            # the same window size on the ST6 recipe (1200x900 / 3 = 400x300)
            line["adjoint_st6"] = adjoint_window(dev, max(3, args.warmup), passes=12, scale=1.0 / 3.0, name="c1")
        print(json.dumps(line), flush=True)
    m.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
