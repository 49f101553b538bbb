#!/usr/bin/env python
"""Throughput of the point-source model-map path on B200, surrogate and plain.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2] [--impl ours|reference]

Metric (one line, printed by rank 0): srcmap pixels/s at 1e-4 relative error
of the learned surrogate with its plain-cubature fallback, next to the plain GPU
cubature path on the same B200.  One srcmap pixel is one (source, x, y, energy)
element of the [S, H, W, E] model map.  One step = one pass of the hot path
over the whole workload: exposure -> mean PSF -> source maps (the three calls of
the reference's main.cxx:28-30) for every source, inputs resident in HBM.

  value        surrogate-plus-fallback path (network where its calibrated error
               cells allow, FP64 12-point rule elsewhere, every 16th pixel
               checked), CUDA-graph replay
  plain_value  the plain path (12-point rule for every value), CUDA-graph replay
  e2e          the surrogate path through the public call from pinned host
               buffers to a pinned host map (copies inside the timed region)

Workload: config c2 by default (500 point sources, 10 % within 1 deg of the
map edge, CAR 400x400 @ 0.05 deg, 37 energies 100 MeV - 1 TeV, livetime cube
nside 64 x 40), seeded synthetic inputs.  The line also carries c4 (2000
sources, 800x800, 50 energies) run in chunks of sources, the FP64-output plain
path, the FP64 oracle's errors of both paths on sampled sources, and the CPU
reference timed on the host cores.

For N > 1 (torchrun, or --gpus N which launches it) every rank runs its own
job of the same size (sources are independent; no collective on the data
path): weak scaling, value = all ranks' pixels / the slowest rank's time.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "srcmap pixels/sec at 1e-4 rel err: NN surrogate vs plain GPU cubature, 1 B200"
UNIT = "srcmap pixels/s (pixel = one (source, x, y, energy) element)"
CHECK_TOL = 1e-4


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c2", choices=["c0", "c1", "c2", "c4"])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--sources", type=int, default=0,
                    help="sources per GPU instead of the configuration's (a smaller case for profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="time eager launches instead of CUDA graphs")
    ap.add_argument("--no-adaptive", action="store_true", help="skip the adaptive-cubature measurement")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="time only the plain path (value is then the plain path's)")
    ap.add_argument("--no-c4", action="store_true", help="skip the chunked c4 measurement")
    ap.add_argument("--no-f64", action="store_true", help="skip the FP64-output plain path")
    ap.add_argument("--no-cutouts", action="store_true", help="skip the c2 per-source cutout measurement")
    ap.add_argument("--no-oracle", action="store_true", help="skip the FP64 oracle error on sampled sources")
    ap.add_argument("--no-tune", action="store_true", help="keep the library's default launch shapes")
    ap.add_argument("--surrogate-samples", type=int, default=10_000_000)
    ap.add_argument("--surrogate-epochs", type=int, default=60)
    ap.add_argument("--surrogate-file", default="",
                    help="load the trained, calibrated network from this file if it exists (no training "
                         "launches: for a profiler's launch list), else train it and save it there")
    ap.add_argument("--cell-margin", type=float, default=0.7,
                    help="the network serves error cells whose held-out worst error is below margin x 1e-4")
    ap.add_argument("--exposure-map-nside", type=int, default=0,
                    help="time only the full-sky exposure map at this nside and exit")
    ap.add_argument("--kernel", default="windows", choices=["windows", "cuda_cores", "tcgen05"],
                    help="FP32 source-map write pass of the plain path")
    return ap.parse_args()


def load_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return {}


def sample_sources(S: int, n: int) -> np.ndarray:
    """n source indices spread over 0..S-1 (the first and last included)."""
    n = max(1, min(S, n))
    return np.unique(np.linspace(0, S - 1, n).round().astype(np.int64))


def env_rank():
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self, t0: float, t1: float):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9 and p[1].replace(".", "").isdigit():
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm = [float(r[1]) for r in rows]
        busy = [float(r[1]) for r in rows if float(r[3] or 0) > 200.0] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": float(rows[0][2]),
                "reasons": reasons, "samples": len(rows), "power_w_max": max(float(r[3] or 0) for r in rows)}


# ----------------------------------------------------------------------------- device inputs
def to_device_job(job, torch, dev):
    """Device-resident copies of every input of the three calls."""
    from xtsrcmaps_b200.api import ExpCube
    from xtsrcmaps_b200.irf import IrfGrid

    t = lambda a, dt=torch.float64: torch.as_tensor(np.asarray(a), device=dev).to(dt).contiguous()

    def grid(g):
        return IrfGrid(t(g.cosths), t(g.logEs), t(g.params), g.min_cos_theta)

    return dict(
        cube=ExpCube(t(job.exp_cube.cosbins, torch.float32), job.exp_cube.nside, 40,
                     job.exp_cube.cosmin, job.exp_cube.thetabin),
        wcube=ExpCube(t(job.wexp_cube.cosbins, torch.float32), job.wexp_cube.nside, 40,
                      job.wexp_cube.cosmin, job.wexp_cube.thetabin),
        logEs=t(job.logEs), src=t(job.src_sph), af=grid(job.aeff_front), ab=grid(job.aeff_back))


def pinned_job(job, torch):
    """Host copies of the step inputs in pinned (page-locked) memory."""
    from xtsrcmaps_b200.api import ExpCube

    def pin(a, dt=None):
        a = np.ascontiguousarray(a if dt is None else np.asarray(a, dt))
        return torch.from_numpy(a).pin_memory().numpy()

    return dict(
        cube=ExpCube(pin(job.exp_cube.cosbins), job.exp_cube.nside, 40, job.exp_cube.cosmin, job.exp_cube.thetabin),
        wcube=ExpCube(pin(job.wexp_cube.cosbins), job.wexp_cube.nside, 40, job.wexp_cube.cosmin, job.wexp_cube.thetabin),
        logEs=pin(job.logEs, np.float64), src=pin(job.src_sph, np.float64))

# ----------------------------------------------------------------------------- our arm
class Stepper:
    """Warm-up, optional CUDA-graph capture and CUDA-event timing of one step
    function on one stream, with an L2 flush (a 256 MiB write) between timed
    steps outside the events."""

    def __init__(self, torch, stream, dev, flush, use_graph: bool):
        self.torch, self.stream, self.dev, self.flush, self.use_graph = torch, stream, dev, flush, use_graph

    def capture(self, fn, warmup: int, profiled: bool = False):
        from xtsrcmaps_b200 import api as A

        torch = self.torch
        A.profile_enable(True, keep=True) if profiled else A.profile_enable(False)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            fn()
        for _ in range(max(3, warmup)):
            with torch.cuda.stream(self.stream):
                g.replay()
        torch.cuda.synchronize(self.dev)
        if profiled:
            A.profile_read()

        def run():
            with torch.cuda.stream(self.stream):
                g.replay()
        run.graph = g
        return run

    def time(self, run, steps: int, dist=None, per_step=None) -> float:
        torch = self.torch
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        torch.cuda.synchronize(self.dev)
        if dist:
            dist.barrier()
        for k in range(steps):
            with torch.cuda.stream(self.stream):
                self.flush.zero_()
            evs[k][0].record(self.stream)
            run()
            evs[k][1].record(self.stream)
            if per_step:
                self.stream.synchronize()
                per_step()
        torch.cuda.synchronize(self.dev)
        return sum(a.elapsed_time(b) for a, b in evs)


def train_surrogate(args, A, dev, log=None):
    """The learned surrogate, trained on the GPU (untimed) on 12-point-rule
    samples of a c2-style job of another seed (separations log-uniform in
    0.001-30 deg, pixel sizes 0.025-0.2 deg), its error cells calibrated on a
    held-out sample of a third seed, and its error on a fourth against the
    centre value alone."""
    import torch

    from xtsrcmaps_b200.surrogate import Surrogate, samples
    from xtsrcmaps_b200.synth import make_job

    def tables(seed):
        j = make_job("c2", seed=seed)
        lt = A.livetime_efficiency_factors(j.logEs, j.effic_front)
        f = A.normalize_rpsf(j.rpsf_front, j.scale_front)
        b = A.normalize_rpsf(j.rpsf_back, j.scale_back)
        ex = A.compute_exposure(j.exp_cube, j.wexp_cube, j.logEs, j.src_sph, j.aeff_front, j.aeff_back, lt)
        ps = A.compute_psf_data(f, b, ex, j.logEs, lt)
        return j, torch.as_tensor(np.ascontiguousarray(ps.uPsf), device=dev)

    tj, tu = tables(args.seed + 100)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    X, Y = samples(tu, tj.logEs, args.surrogate_samples, seed=args.seed + 1)
    net = Surrogate(device=dev, seed=args.seed)
    losses = net.train(X, Y, epochs=args.surrogate_epochs)
    torch.cuda.synchronize(dev)
    t_train = time.perf_counter() - t0
    del X, Y
    cj, cu = tables(args.seed + 200)
    Xc, Yc = samples(cu, cj.logEs, 4_000_000, seed=args.seed + 2)
    cal = net.calibrate(Xc, Yc, tol=CHECK_TOL, margin=args.cell_margin)
    del Xc, Yc
    hj, hu = tables(args.seed + 300)
    Xh, Yh = samples(hu, hj.logEs, 1_000_000, seed=args.seed + 3)
    yp = net.predict(Xh)
    rho = 10.0 ** Xh[:, 0].double()
    far = rho >= 30.0  # where a surrogate of this kind can serve; nearer pixels take the rule
    err_net = ((yp.double() - Yh.double()).abs() / rho ** 2)[far]
    err_c = (Yh.double().abs() / rho ** 2)[far]
    held = {"samples": int(Xh.shape[0]), "samples_rho_ge_30": int(far.sum()),
            "rms_rel_err": float(err_net.pow(2).mean().sqrt()),
            "frac_within_1e-4": float((err_net <= 1e-4).double().mean()),
            "centre_value_rms_rel_err": float(err_c.pow(2).mean().sqrt()),
            "note": "relative error of the pixel mean over held-out samples with rho >= 30"}
    held["gain_rms"] = held["centre_value_rms_rel_err"] / held["rms_rel_err"]
    train = {"samples": args.surrogate_samples, "epochs": args.surrogate_epochs, "seconds": t_train,
             "first_epoch_loss": losses[0], "final_loss": losses[-1],
             "sample_range": "separations log-uniform 0.001-30 deg, pixel sizes 0.025-0.2 deg, c2-style mean PSFs "
                             "(500 sources) of another seed",
             "calibration": cal, "held_out": held}
    return net, train


def oracle_errors(job, idx, maps: dict) -> dict:
    """Largest relative error of each map [S, H, W, E] (CUDA tensor or numpy) over
    the sources ``idx`` against the FP64 oracle of those sources."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import copy

    from helpers import oracle_pipeline

    sub = copy.copy(job)
    sub.src_sph = job.src_sph[idx]
    ref = oracle_pipeline(sub)["map"]
    out = {}
    for name, m in maps.items():
        got = m[idx]
        got = got.cpu().numpy() if hasattr(got, "cpu") else np.asarray(got)
        err = np.abs(got.astype(np.float64) - ref) / np.maximum(np.abs(ref), 1e-300)
        out[name] = {"max_rel_err": float(err.max()), "frac_within_1e-4": float((err <= 1e-4).mean()),
                     "frac_within_1e-5": float((err <= 1e-5).mean())}
    return out


def rel_err_between(a, b, torch) -> dict:
    """Largest relative difference of map a from map b over every value, by source."""
    worst, within = 0.0, 0
    for s in range(a.shape[0]):
        d = (a[s].double() - b[s].double()).abs() / b[s].double().abs().clamp_min(1e-300)
        worst = max(worst, float(d.max()))
        within += int((d <= 1e-4).sum())
    return {"max_rel_err": worst, "frac_within_1e-4": within / a.numel()}


def run_ours(args, rank, world, local_rank):
    import torch

    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200.irf import IrfGrid
    from xtsrcmaps_b200.shard import shard_sources
    from xtsrcmaps_b200.synth import CONFIGS, DESCRIPTIONS, make_job

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    A.init(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    # one global source list, CONFIGS[config]["S"] sources per GPU, sharded over the
    # ranks (weak scaling); every rank holds the same livetime cube and IRFs
    per_gpu = args.sources if args.sources > 0 else CONFIGS[args.config]["S"]
    job = make_job(args.config, seed=args.seed, n_sources=per_gpu * world)
    job.src_sph = job.src_sph[shard_sources(job.S, world)[rank]]
    S, H, W, E = job.S, job.wcs.naxis1, job.wcs.naxis2, job.E
    n_values = job.n_values
    # IRF set-up (Irf::collect_irf_data, untimed like the reference's ingest)
    ltf_h = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf_h = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb_h = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    d = to_device_job(job, torch, dev)
    tt = lambda a: torch.as_tensor(np.asarray(a), device=dev, dtype=torch.float64)
    nf = IrfGrid(tt(nf_h.cosths), tt(nf_h.logEs), tt(nf_h.params), nf_h.min_cos_theta)
    nb = IrfGrid(tt(nb_h.cosths), tt(nb_h.logEs), tt(nb_h.params), nb_h.min_cos_theta)
    ltf = tt(ltf_h)
    out = torch.empty((S, H, W, E), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    stream = torch.cuda.Stream(dev)
    stepper = Stepper(torch, stream, dev, flush, not args.no_graph)
    peaks = load_peaks()
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    tensor_peak = peaks.get("bf16_tflops", 1590.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"

    net, train = (None, None)
    if not args.no_surrogate:
        if args.surrogate_file and os.path.exists(args.surrogate_file):
            from xtsrcmaps_b200.surrogate import Surrogate

            net = Surrogate.load(args.surrogate_file, device=dev)
            train = {"loaded": args.surrogate_file}
        else:
            net, train = train_surrogate(args, A, dev)
            if args.surrogate_file:
                net.save(args.surrogate_file)

    # launch shapes by measurement on this job (window-pass, write-pass and
    # network blocks per SM), set for everything timed below
    from xtsrcmaps_b200.autotune import tune_launch_shapes

    shapes = {"choice": "library defaults (--no-tune)", "ms": {}}
    if not args.no_tune:
        with torch.cuda.stream(stream):
            ex_t = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps_t = A.compute_psf_data(nf, nb, ex_t, d["logEs"], ltf)
            shapes = tune_launch_shapes(job.wcs, d["src"], ex_t.exposure, ps_t.uPsf, ps_t.partial_psf_integral,
                                        net=net)
        del ex_t, ps_t

    # one plain step = the public call that replaces main.cxx:28-30 (point_source_maps:
    # exposure, mean PSF and model maps; the map geometry runs on a second stream
    # beside exposure and PSF)
    def step_plain():
        with torch.cuda.stream(stream):
            A.point_source_maps(job.wcs, d["src"], d["cube"], d["wcube"], d["logEs"], d["af"], d["ab"], nf, nb,
                                ltf, out=out, with_info=False, kernel=args.kernel)

    out_s = torch.empty_like(out) if net is not None else None

    # one surrogate step: the same three calls with the surrogate's model map
    def step_sur():
        with torch.cuda.stream(stream):
            ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
            A.point_src_model_map_wcs_surrogate(job.wcs, d["src"], ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                                d["logEs"], net, check_tol=CHECK_TOL, with_info=False, out=out_s,
                                                stats=False)

    steps = [("plain", step_plain)] + ([("surrogate", step_sur)] if net is not None else [])
    for _ in range(max(3, args.warmup)):
        for _, fn in steps:
            fn()
    torch.cuda.synchronize(dev)
    runs, prof_runs = {}, {}
    launch = "eager launches"
    if stepper.use_graph:
        try:
            for name, fn in steps:
                runs[name] = stepper.capture(fn, args.warmup)
            launch = "one CUDA graph per step (each path captured once)"
        except Exception as exc:  # capture refused: both paths eager
            runs, prof_runs = {}, {}
            launch = "eager launches (graph capture failed: %s)" % str(exc).splitlines()[0][:120]
            A.profile_enable(False)
            torch.cuda.synchronize(dev)
    for name, fn in steps:
        runs.setdefault(name, fn)

    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    ms = {name: stepper.time(runs[name], args.steps, dist) for name, _ in steps}
    ck = clocks.stop(0, 0)
    A.profile_enable(False)
    sur_stats = None
    if net is not None:
        from xtsrcmaps_b200.surrogate import last_stats

        with torch.cuda.stream(stream):
            sur_stats = last_stats(dev)

    # per-kernel times: the instrumented graphs (their timers were recorded at capture
    # and are kept), read after every replay; eager: the profiler on during extra steps
    prof = {}
    for name, fn in steps:
        p = {}

        def add(pp, p=p):
            for k_, (n_, t_) in pp.items():
                a_ = p.get(k_, (0, 0.0))
                p[k_] = (a_[0] + n_, a_[1] + t_)

        if stepper.use_graph and launch.startswith("one CUDA graph"):
            # an instrumented graph of this path, captured and read before the next one:
            # enabling or disabling the library's timers clears their records
            prof_runs[name] = stepper.capture(fn, args.warmup, profiled=True)
            msp = stepper.time(prof_runs[name], args.steps, None, lambda: add(A.profile_read()))
            A.profile_enable(False)
        else:
            A.profile_enable(True)
            msp = stepper.time(fn, args.steps, None, lambda: add(A.profile_read()))
            A.profile_enable(False)
        prof[name] = (p, msp)
    A.profile_enable(False)

    def ms_max(m):
        t = torch.tensor([m], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ms = {k: ms_max(v) for k, v in ms.items()}
    val = {k: n_values * world * args.steps / (v * 1e-3) for k, v in ms.items()}
    head = "surrogate" if net is not None else "plain"

    def kernels_of(name):
        p, _ = prof[name]
        return {k: {"launches": v[0], "ms": round(v[1], 4)} for k, v in p.items()}

    def dominant_of(name):
        p, msp = prof[name]
        if not p:
            return None
        k, (n, t) = max(p.items(), key=lambda kv: kv[1][1])
        return {"kernel": k, "share": t / msp if msp else None, "avg_launch_ms": t / n if n else None,
                "launches_per_step": n / args.steps}

    # roofline of the write pass of the plain path (the kernel that writes the srcmap
    # values): algorithmic bytes per launch over its CUDA-event launch time
    epad = (E + 3) // 4 * 4
    p_plain, msp_plain = prof["plain"]
    kn, kms = p_plain.get("k_srcmap", (0, 0.0))
    per_step = kn / args.steps if kn else 1
    alg_bytes = (4 * n_values + 4 * S * 401 * epad + 24 * (H + 1) * (W + 1) + 8 * H * W) / per_step
    achieved = alg_bytes / (kms / kn * 1e-3) / 1e9 if kn else None
    traffic, traffic_note = None, None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "k_srcmap_traffic.json")))
        if args.kernel == "windows" and tr.get("dram_bytes_per_launch"):
            # captured on a smaller case (c2's map with 50 sources: 296 M values per
            # launch); the write pass's DRAM traffic grows with the values it writes, so it
            # is scaled to this launch's values
            ref_values = tr["values"]
            traffic = tr["dram_bytes_per_launch"] * (n_values / per_step) / ref_values
            traffic_note = (f"ncu DRAM bytes of one launch on {tr['workload']} ({tr['dram_bytes_per_launch']} B "
                            f"for {ref_values} values), scaled by values written")
    except (OSError, ValueError, KeyError):
        pass
    roof_write = {"bound": "hbm", "kernel": "k_srcmap", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                  "frac": (achieved / hbm_peak) if achieved else None, "peak_source": peak_src, "traffic": traffic,
                  "traffic_source": traffic_note,
                  "alg_bytes_per_launch": int(alg_bytes), "launches_per_step": per_step,
                  "avg_launch_ms": kms / kn if kn else None,
                  "note": "write pass of the plain path: 4 B per srcmap value + the scaled tables + geometry"}
    path_gbs = {k: 4.0 * n_values * world / (v / args.steps * 1e-3) / 1e9 for k, v in ms.items()}
    roofline_plain_path = {"bound": "hbm", "achieved": path_gbs["plain"], "peak": hbm_peak, "unit": "GB/s",
                           "frac": path_gbs["plain"] / hbm_peak,
                           "note": "whole plain step: 4 B written per srcmap value over the step time"}
    roofline = roof_write
    if net is not None:
        # the surrogate step's dominant kernel: the network's forward pass on tcgen05
        p_s, msp_s = prof["surrogate"]
        # the network's inference launches: the four-tile kernel (default) or the
        # two-warpgroup kernel (mlp_blocks_per_sm 1 or 2)
        kname = "k_mlp_infer" if "k_mlp_infer" in p_s else "k_mlp_forward"
        fn_, fms = p_s.get(kname, (0, 0.0))
        rows = (sur_stats or {}).get("evaluated", 0)
        flop = 2 * (5 * 128 + 2 * 128 * 128 + 128) * rows
        tflops = flop / (fms / args.steps * 1e-3) / 1e12 if fms else None
        # DRAM traffic per launch from the committed ncu capture of the kernel, scaled by
        # the rows of an average launch here (the traffic is the rows' features and outputs)
        m_traffic, m_note = None, None
        try:
            tm = json.load(open(os.path.join(ROOT, "profiles", "k_mlp_infer_traffic.json")))
            if kname == tm["kernel"] and fn_:
                m_traffic = tm["dram_bytes_per_launch"] * (rows / (fn_ / args.steps)) / tm["rows"]
                m_note = (f"ncu DRAM bytes of one launch over {tm['rows']} rows ({tm['dram_bytes_per_launch']} B), "
                          "scaled by this step's rows per launch")
        except (OSError, KeyError, ValueError):
            pass
        roofline = {"bound": "tensor", "kernel": kname, "achieved": tflops, "peak": tensor_peak,
                    "unit": "TFLOP/s", "frac": tflops / tensor_peak if tflops else None, "peak_source": peak_src,
                    "traffic": m_traffic, "traffic_source": m_note,
                    "alg_flops_per_step": flop, "launches_per_step": fn_ / args.steps,
                    "avg_launch_ms": fms / fn_ if fn_ else None,
                    "note": "67,072 FLOP per network row (5-128-128-128-1, hidden layers on tcgen05 BF16 with "
                            "FP32 accumulation); rows = values the network evaluated per step"}
    gpu_launches = sum(v[0] for v in prof[head][0].values())

    # accuracy: the FP64 oracle on sampled sources (rank 0), and the surrogate map
    # against the plain map over every value
    errors = None
    if rank == 0 and not args.no_oracle:
        idx = sample_sources(S, 16)
        maps = {"plain": out}
        if net is not None:
            maps["surrogate"] = out_s
        errors = oracle_errors(job, idx, maps)
        errors["sources"] = [int(i) for i in idx]
        if net is not None:
            errors["surrogate_vs_plain_all_values"] = rel_err_between(out_s, out, torch)

    # end to end through the public API with host (pinned) buffers
    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(args, A, job, nf_h, nb_h, ltf_h, net, torch, dev, dist, world, n_values)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(job)

    # the plain path with FP64 maps (XTS_OUT_F64): the reference's output precision
    f64 = None
    if not args.no_f64 and world == 1:
        f64 = measure_f64(args, A, job, d, nf, nb, ltf, stepper, torch, dev, n_values, out, rank)

    adaptive = None
    if not args.no_adaptive and world == 1:
        adaptive = measure_adaptive(args, A, job, d, nf, nb, ltf, stepper, torch, dev, n_values)

    from xtsrcmaps_b200.autotune import tune_write_pass

    with torch.cuda.stream(stream):
        ex_t = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
        ps_t = A.compute_psf_data(nf, nb, ex_t, d["logEs"], ltf)
        autotune = tune_write_pass(job.wcs, d["src"], ex_t.exposure, ps_t.uPsf, ps_t.partial_psf_integral)

    cutouts = None
    if args.config == "c2" and not args.no_cutouts and world == 1:
        cutouts = measure_cutouts(args, A, job, d, nf, nb, ltf, stepper, torch, dev, rank)

    c4 = None
    if args.config == "c2" and not args.no_c4 and world == 1:
        del out_s
        out = None
        torch.cuda.empty_cache()
        c4 = measure_c4(args, A, net, torch, dev, stream, flush, rank)

    runs = prof_runs = None  # release the captured graphs before the process group goes away
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    surrogate = None
    if net is not None:
        served = (sur_stats["accepted"] / sur_stats["values"]) if sur_stats and sur_stats["values"] else 0.0
        surrogate = {"stats": sur_stats, "served_frac": served, "check_tol": CHECK_TOL, "check_every": 16,
                     "train": train, "kernels": kernels_of("surrogate"), "dominant_kernel": dominant_of("surrogate")}
    line = {
        "metric": METRIC, "value": val[head], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms[head] / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 maps (FP64 separations, chord offsets from the FP64 pixel-centre chord, FP64 sums and "
                 "tables; network BF16 with FP32 accumulation)",
        "data": "synthetic (seeded livetime cube, IRF tables and source positions; no public dataset)",
        "config": {"workload": args.config + ": " + DESCRIPTIONS[args.config]
                   + (f" (reduced to {S} sources per GPU)" if args.sources > 0 else ""), "sources_per_gpu": S,
                   "map": f"{H}x{W}", "energies": E, "values_per_step_per_gpu": n_values,
                   "parallelism": f"sources sharded over {world} GPU(s), no data-path collective",
                   "l2": "256 MiB buffer written between timed steps (L2 flush); the map written per step "
                         f"({4 * n_values / 1e9:.1f} GB) also exceeds the 126 MB L2",
                   "output_dtype": "float32", "launch": launch, "headline_path": head},
        "plain_value": val["plain"], "plain_ms_per_step": ms["plain"] / args.steps,
        "surrogate_vs_plain": (val[head] / val["plain"]) if net is not None else None,
        "source_pixel_rates": {"unit": "(source, pixel) pairs/s (all E energies of a pixel)",
                               "value": val[head] / E, "plain": val["plain"] / E},
        "roofline": roofline, "roofline_write_pass": roof_write, "roofline_plain_path": roofline_plain_path,
        "dominant_kernel": dominant_of(head), "dominant_kernel_plain": dominant_of("plain"),
        "kernels": kernels_of(head), "kernels_plain": kernels_of("plain"), "gpu_launches": gpu_launches,
        "clocks": ck, "e2e": e2e, "cpu_baseline": cpu, "errors_vs_fp64_oracle": errors,
        "surrogate": surrogate, "f64": f64, "c2_cutouts": cutouts, "c4": c4, "adaptive": adaptive,
        "autotune_launch_shapes": shapes, "autotune_write_pass": autotune,
    }
    print(json.dumps(line), flush=True)


def measure_e2e(args, A, job, nf_h, nb_h, ltf_h, net, torch, dev, dist, world, n_values):
    """The headline path end to end through the public call, from pinned host
    inputs to a pinned host map; and the plain fused call the same way."""
    hp = pinned_job(job, torch)
    S, H, W, E = job.S, job.wcs.naxis1, job.wcs.naxis2, job.E
    hout = torch.empty((S, H, W, E), dtype=torch.float32).pin_memory()
    hout_np = hout.numpy()
    ke = max(3, min(args.steps, 10))

    def wall(fn):
        for _ in range(3):
            fn()
        if dist:
            dist.barrier()
        t0_ = time.perf_counter()
        for _ in range(ke):
            fn()
        te_t = torch.tensor([time.perf_counter() - t0_], dtype=torch.float64, device=dev)
        if dist:
            dist.all_reduce(te_t, op=dist.ReduceOp.MAX)
        return float(te_t.item())

    def step_plain():
        A.point_source_maps(job.wcs, hp["src"], hp["cube"], hp["wcube"], hp["logEs"], job.aeff_front,
                            job.aeff_back, nf_h, nb_h, ltf_h, out=hout_np, with_info=False, kernel=args.kernel)

    C_ = int(job.exp_cube.nbrbins)
    grid_b = lambda g: 8 * (g.cosths.size + g.logEs.size + g.params.size)
    grids = grid_b(job.aeff_front) + grid_b(job.aeff_back) + grid_b(nf_h) + grid_b(nb_h)
    te_p = wall(step_plain)
    plain = {"value": n_values * world * ke / te_p, "unit": UNIT,
             "h2d_bytes_per_step": int(2 * 4 * S * C_ + 8 * E + 16 * S + grids + 16 * E),
             "d2h_bytes_per_step": int(4 * n_values + 8 * S), "steps": ke,
             "note": "point_source_maps (the three calls of main.cxx:28-30 fused, plain cubature) from pinned host "
                     "buffers to a pinned host map; the library uploads only the livetime rows at the sources' "
                     "pixels and copies the map out by chunks of sources while later chunks compute"}
    if net is None:
        return plain
    hcube = torch.from_numpy(np.ascontiguousarray(job.exp_cube.cosbins)).pin_memory()
    hwcube = torch.from_numpy(np.ascontiguousarray(job.wexp_cube.cosbins)).pin_memory()
    from xtsrcmaps_b200.api import ExpCube

    cube = ExpCube(hcube, job.exp_cube.nside, 40, job.exp_cube.cosmin, job.exp_cube.thetabin)
    wcube = ExpCube(hwcube, job.wexp_cube.nside, 40, job.wexp_cube.cosmin, job.wexp_cube.thetabin)
    src = torch.from_numpy(np.ascontiguousarray(job.src_sph, dtype=np.float64)).pin_memory()
    le = torch.from_numpy(np.ascontiguousarray(job.logEs, dtype=np.float64)).pin_memory()

    def step_sur():
        A.point_source_maps_surrogate(job.wcs, src, cube, wcube, le, job.aeff_front, job.aeff_back, nf_h, nb_h,
                                      ltf_h, net, check_tol=CHECK_TOL, out=hout, with_info=False, stats=False)

    te_s = wall(step_sur)
    return {"value": n_values * world * ke / te_s, "unit": UNIT,
            "h2d_bytes_per_step": int(2 * 4 * S * C_ + 8 * E + 16 * S + grids + 16 * E),
            "d2h_bytes_per_step": int(4 * n_values), "steps": ke,
            "note": "point_source_maps_surrogate (the three calls of main.cxx:28-30 fused, surrogate model map) "
                    "from pinned host buffers to a pinned host map, copies inside the timed region; the library "
                    "uploads only the livetime rows at the sources' pixels and copies the map out by groups of "
                    "sources while later groups compute",
            "plain": plain}


def measure_f64(args, A, job, d, nf, nb, ltf, stepper, torch, dev, n_values, out32, rank):
    """The plain path writing FP64 maps (XTS_OUT_F64, the reference's output type:
    the reference's per-point FP64 arithmetic throughout), timed as the FP32 path."""
    S, H, W, E = job.S, job.wcs.naxis1, job.wcs.naxis2, job.E
    out = torch.empty((S, H, W, E), dtype=torch.float64, device=dev)

    def step():
        with torch.cuda.stream(stepper.stream):
            A.point_source_maps(job.wcs, d["src"], d["cube"], d["wcube"], d["logEs"], d["af"], d["ab"], nf, nb,
                                ltf, out_dtype="float64", out=out, with_info=False)

    for _ in range(3):
        step()
    k = max(3, min(args.steps, 10))
    ms = stepper.time(step, k)
    res = {"value": n_values * k / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k,
           "launch": "eager launches", "output_dtype": "float64",
           "hbm_gbs": 8.0 * n_values / (ms / k * 1e-3) / 1e9}
    if rank == 0 and not args.no_oracle:
        idx = sample_sources(S, 4)
        res["errors_vs_fp64_oracle"] = oracle_errors(job, idx, {"f64": out})["f64"]
        res["errors_vs_fp64_oracle"]["sources"] = [int(i) for i in idx]
    del out
    torch.cuda.empty_cache()
    return res


def measure_cutouts(args, A, job, d, nf, nb, ltf, stepper, torch, dev, rank):
    """c2 with its per-source cutout radii (2-15 deg): every source's map is its
    window of the map (ragged output), the plain path's window and write passes
    each one persistent launch over a work queue of (source, tile) items; exposure,
    mean PSF and cutout maps captured in one CUDA graph per step; the FP64 oracle of
    the same windows on sampled sources."""
    cut, total = A.cutout_windows(job.wcs, job.src_sph, job.cutout_deg)
    E = job.E
    cut_d = torch.as_tensor(np.frombuffer(cut.tobytes(), dtype=np.uint8).copy(), device=dev)
    out = torch.empty((total, E), dtype=torch.float32, device=dev)

    def step():
        with torch.cuda.stream(stepper.stream):
            ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
            A.point_src_model_map_cutouts(job.wcs, d["src"], cut_d, ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                          out=out, with_info=False)

    for _ in range(3):
        step()
    torch.cuda.synchronize(dev)
    launch = "eager launches"
    run = step
    if stepper.use_graph:
        try:
            run = stepper.capture(step, args.warmup)
            launch = "one CUDA graph per step"
        except Exception as exc:
            launch = "eager launches (graph capture failed: %s)" % str(exc).splitlines()[0][:120]
    k = max(3, min(args.steps, 10))
    ms = stepper.time(run, k)
    nv = total * E
    res = {"workload": "c2 with per-source cutouts (radii uniform 2-15 deg): source s's map is its window of the "
                       "map, the reference's model map of that sub-map",
           "value": nv / (ms / k * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k, "launch": launch,
           "values_per_step": nv, "dense_values": job.n_values, "pixels": total,
           "hbm_gbs": 4.0 * nv / (ms / k * 1e-3) / 1e9}
    if rank == 0 and not args.no_oracle:
        from oracle import oracle as O

        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import copy

        from helpers import oracle_pipeline

        idx = sample_sources(job.S, 8)
        sub = copy.copy(job)
        sub.src_sph = job.src_sph[idx]
        r = oracle_pipeline(sub, with_map=False)
        sc = cut[idx].copy()
        sc["offset"] = np.concatenate([[0], np.cumsum(sc["nh"].astype(np.int64) * sc["nw"])[:-1]])
        ref = O.point_src_model_map_cutouts(job.wcs, sub.src_sph, sc, r["exposure"], r["upsf"], r["partial"])
        g = out.cpu().numpy()
        worst = 0.0
        for k_, s in enumerate(idx):
            n = int(cut[s]["nh"]) * int(cut[s]["nw"])
            if n:
                a = g[int(cut[s]["offset"]):int(cut[s]["offset"]) + n].astype(np.float64)
                b = ref["map"][int(sc[k_]["offset"]):int(sc[k_]["offset"]) + n]
                worst = max(worst, float((np.abs(a - b) / np.maximum(np.abs(b), 1e-300)).max()))
        res["errors_vs_fp64_oracle"] = {"max_rel_err": worst, "sources": [int(i) for i in idx]}
    del out
    torch.cuda.empty_cache()
    return res


def measure_adaptive(args, A, job, d, nf, nb, ltf, stepper, torch, dev, n_values):
    """The pipeline with adaptive Genz-Malik cubature of each pixel (rtol 1e-4,
    depth 6) in place of the 12-point rule, eager launches."""
    out_a = torch.empty((job.S, job.wcs.naxis1, job.wcs.naxis2, job.E), dtype=torch.float32, device=dev)

    def step():
        with torch.cuda.stream(stepper.stream):
            ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
            A.point_src_model_map_wcs_adaptive(job.wcs, d["src"], ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                               rtol=1e-4, max_depth=6, out=out_a, with_info=False)

    for _ in range(3):
        step()
    k = max(3, min(args.steps, 5))
    ms = stepper.time(step, k)
    del out_a
    torch.cuda.empty_cache()
    return {"value": n_values / (ms / k * 1e-3), "unit": UNIT, "ms_per_step": ms / k, "steps": k, "rtol": 1e-4,
            "max_depth": 6, "note": "point_src_model_map_wcs_adaptive (Genz-Malik 7/5 per pixel) in place of the "
                                    "12-point rule; eager launches"}


def measure_c4(args, A, net, torch, dev, stream, flush, rank, chunk: int = 250):
    """Config c4 (2000 sources, CAR 800x800 @ 0.025 deg, 50 energies, nside 128):
    256 GB of FP32 maps do not fit on one GPU, so each step runs the sources in
    chunks of ``chunk`` through the public calls, every chunk's maps overwriting
    the previous chunk's in one device buffer (nothing is copied out); plain and
    surrogate paths, eager launches, and the FP64 oracle on two sampled sources."""
    from xtsrcmaps_b200.irf import IrfGrid
    from xtsrcmaps_b200.synth import DESCRIPTIONS, make_job

    job = make_job("c4", seed=args.seed)
    S, H, W, E = job.S, job.wcs.naxis1, job.wcs.naxis2, job.E
    ltf_h = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf_h = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb_h = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    d = to_device_job(job, torch, dev)
    tt = lambda a: torch.as_tensor(np.asarray(a), device=dev, dtype=torch.float64)
    nf = IrfGrid(tt(nf_h.cosths), tt(nf_h.logEs), tt(nf_h.params), nf_h.min_cos_theta)
    nb = IrfGrid(tt(nb_h.cosths), tt(nb_h.logEs), tt(nb_h.params), nb_h.min_cos_theta)
    ltf = tt(ltf_h)
    buf = torch.empty((chunk, H, W, E), dtype=torch.float32, device=dev)
    chunks = [(s0, min(S, s0 + chunk)) for s0 in range(0, S, chunk)]
    stepper = Stepper(torch, stream, dev, flush, False)

    def plain(keep=None):
        with torch.cuda.stream(stream):
            for s0, s1 in chunks:
                A.point_source_maps(job.wcs, d["src"][s0:s1], d["cube"], d["wcube"], d["logEs"], d["af"], d["ab"],
                                    nf, nb, ltf, out=buf[: s1 - s0], with_info=False)
                if keep is not None:
                    keep(s0, s1)

    def sur(keep=None):
        with torch.cuda.stream(stream):
            for s0, s1 in chunks:
                src = d["src"][s0:s1]
                ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], src, d["af"], d["ab"], ltf)
                ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
                A.point_src_model_map_wcs_surrogate(job.wcs, src, ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                                    d["logEs"], net, check_tol=CHECK_TOL, with_info=False,
                                                    out=buf[: s1 - s0], stats=False)
                if keep is not None:
                    keep(s0, s1)

    idx = sample_sources(S, 2)
    kept = {}

    def keeper(name):
        def keep(s0, s1):
            for i in idx:
                if s0 <= i < s1:
                    kept.setdefault(name, {})[int(i)] = buf[i - s0].cpu()
        return keep

    res = {"workload": "c4: " + DESCRIPTIONS["c4"], "values_per_step": job.n_values, "chunk_sources": chunk,
           "chunks": len(chunks),
           "maps": "each chunk's maps overwrite the previous chunk's in one device buffer (nothing copied out)",
           "launch": "eager launches"}
    plain(keeper("plain"))
    k = max(2, min(args.steps, 3))
    ms = stepper.time(plain, k)
    res["plain_value"] = job.n_values / (ms / k * 1e-3)
    res["plain_ms_per_step"] = ms / k
    if net is not None:
        sur(keeper("surrogate"))
        from xtsrcmaps_b200.surrogate import last_stats

        ks = 2
        ms_s = stepper.time(sur, ks)
        res["value"] = job.n_values / (ms_s * 1e-3 / ks)
        res["ms_per_step"] = ms_s / ks
        res["surrogate_vs_plain"] = res["value"] / res["plain_value"]
        with torch.cuda.stream(stream):
            res["surrogate_stats_last_chunk"] = last_stats(dev)
        if res["surrogate_stats_last_chunk"].get("accepted", 0) == 0:
            res["surrogate_note"] = ("no value served by the network: c4's 0.025 deg CAR pixels have solid angles "
                                     "below the smallest training pixel's (0.025^2 deg^2), so the feature-range "
                                     "check gives every value to the 12-point rule")
    if rank == 0 and not args.no_oracle:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import copy

        from helpers import oracle_pipeline

        sub = copy.copy(job)
        sub.src_sph = job.src_sph[idx]
        ref = oracle_pipeline(sub)["map"]
        errs = {}
        for name, per in kept.items():
            got = np.stack([per[int(i)].numpy() for i in idx]).astype(np.float64)
            e = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
            errs[name] = {"max_rel_err": float(e.max()), "frac_within_1e-4": float((e <= 1e-4).mean())}
        errs["sources"] = [int(i) for i in idx]
        res["errors_vs_fp64_oracle"] = errs
    if rank == 0 and not args.no_cpu_baseline:
        # a c4 source is 3.2e7 values (~6 s of one reference thread), and the reference hands
        # out 16 sources per thread, so any sample that keeps more than one thread busy takes
        # over 90 s: two sources on one thread, one pass, declared as such
        res["cpu_baseline"] = cpu_baseline(job, max_sources=2, warm=False)
    del buf
    torch.cuda.empty_cache()
    return res


# ----------------------------------------------------------------------------- CPU legs
def _oracle_worker(args):
    name, seed, idx = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_pipeline
    from xtsrcmaps_b200.synth import make_job

    job = make_job(name, seed=seed)
    job.src_sph = job.src_sph[idx]
    t0 = time.perf_counter()
    r = oracle_pipeline(job)
    return time.perf_counter() - t0, r["map"].size


def _reference_runner(job):
    """One pass of the CPU reference over ``job``: the reference's own code
    compiled under oracle/_ref when it is there (its OpenMP on every host core),
    else None.  Returns (run, threads, description)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import irf_setup, reference_pipeline
    from oracle import oracle_ref as R

    if not R.available():
        return None, 0, ""
    threads = R.set_threads(os.cpu_count() or 1)
    setup = irf_setup(job)  # Irf::collect_irf_data, outside the timed pass as on the GPU
    busy = min(threads, (job.S + 15) // 16)
    desc = (f"the reference's compiled exposure, mean-PSF and model-map code (oracle/_ref), OpenMP with "
            f"{threads} threads; its source loops use schedule(static, 16), so {busy} thread(s) share "
            f"the {job.S} sources")
    return (lambda times=None: reference_pipeline(job, setup, times=times)), threads, desc


def _source_sample(job, max_sources: int):
    """The bench job restricted to a spread sample of its sources: at most
    max_sources, enough for 16 per host thread (the reference's OpenMP chunk)."""
    import copy

    n = min(job.S, max_sources, 16 * (os.cpu_count() or 1))
    idx = sample_sources(job.S, n)
    sub = copy.copy(job)
    sub.src_sph = job.src_sph[idx]
    return sub


def cpu_baseline(job, max_sources: int = 256, warm: bool = True):
    """The CPU reference (compiled reference code, else the FP64 oracle port) on
    the host cores over a sample of the bench job's sources (a warm pass unless
    warm is False, then timed passes for about 10 s); values/s of the sample.
    cores = the threads that had work: the reference's source loops hand out
    chunks of 16 sources (schedule(static, 16))."""
    sub = _source_sample(job, max_sources)
    run, threads, desc = _reference_runner(sub)
    kind = "reference"
    if run is None:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from helpers import oracle_pipeline

        run, threads, kind = (lambda: oracle_pipeline(sub)), 1, "port"
        desc = "the FP64 oracle (a scalar C restatement of the reference path) on one core"
    else:
        threads = min(threads, (sub.S + 15) // 16)
    if warm:
        run()
    times = {}
    t0 = time.perf_counter()
    reps = 0
    while reps < 1 or (time.perf_counter() - t0 < 10.0 and reps < 20):
        if kind == "reference":
            run(times)
        else:
            run()
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    res = {"value": sub.n_values / dt, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{sub.S} of the job's {job.S} sources ({job.wcs.naxis1}x{job.wcs.naxis2}, {job.E} energies; "
                     f"{sub.n_values:.3g} values) {reps} time(s): {desc}; rate scales with values"}
    if times:
        res["seconds_per_pass"] = {k: v / reps for k, v in times.items()}
    return res


def run_reference(args, rank, world):
    """--impl reference: the CPU reference on this box's host cores (rank 0 only),
    each step a sample of the workload's sources (16 per host thread, the
    reference's OpenMP chunk, at most 256)."""
    if rank != 0:
        return
    from xtsrcmaps_b200.synth import DESCRIPTIONS, make_job

    job = make_job(args.config, seed=args.seed)
    sub = _source_sample(job, 256)
    run, threads, desc = _reference_runner(sub)
    if run is not None:
        kind = "reference"
        run()  # warm-up pass: the reference code has no JIT; this touches its buffers once
        warm = 1
        times = []
        t_all = time.perf_counter()
        for _ in range(args.steps):  # stop after ~60 s
            t0 = time.perf_counter()
            run()
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_all > 60.0:
                break
        sample = (f"per step {sub.S} of the {args.config} job's {job.S} sources ({sub.n_values:.3g} values): "
                  f"{desc}")
    else:  # the oracle port, one process per block of sources
        import multiprocessing as mp

        kind = "port"
        cores = os.cpu_count() or 1
        idx = sample_sources(job.S, min(job.S, cores))
        chunks = [(args.config, args.seed, idx[i::cores]) for i in range(cores)]
        chunks = [c for c in chunks if len(c[2])]
        threads = len(chunks)
        ctx = mp.get_context("spawn")
        with ctx.Pool(len(chunks)) as pool:
            warm = 1
            pool.map(_oracle_worker, chunks)
            times = []
            for _ in range(max(1, min(args.steps, 5))):
                t0 = time.perf_counter()
                pool.map(_oracle_worker, chunks)
                times.append(time.perf_counter() - t0)
        sub.src_sph = job.src_sph[idx]
        sample = f"per step {len(idx)} of the {args.config} job's sources, FP64 oracle over {threads} processes"
    ms = 1e3 * sum(times) / len(times)
    value = sub.n_values / (ms * 1e-3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": len(times), "warmup": warm, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
        "config": {"workload": args.config + ": " + DESCRIPTIONS[args.config]},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_exposure_map(args):
    """--exposure-map-nside N: the full-sky exposure map (tcgen05, 3xTF32) on a
    seeded livetime cube of that nside with the c4 energy grid; one JSON line."""
    import torch

    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200.api import ExpCube
    from xtsrcmaps_b200.synth import make_job

    A.init(0)
    dev = torch.device("cuda", 0)
    job = make_job("c4", seed=args.seed, n_sources=1)
    nside, C = int(args.exposure_map_nside), 40
    npix = 12 * nside * nside
    rng = np.random.default_rng(args.seed)
    cube = (2e5 * rng.lognormal(0.0, 0.2, (npix, C))).astype(np.float32)
    c = ExpCube(torch.as_tensor(cube, device=dev), nside, C, 0.0, True)
    w = ExpCube(torch.as_tensor(0.9 * cube, device=dev), nside, C, 0.0, True)
    ltf = torch.as_tensor(A.livetime_efficiency_factors(job.logEs, job.effic_front), device=dev)
    tg = lambda g: type(g)(*[torch.as_tensor(np.asarray(v), device=dev) if isinstance(v, np.ndarray) else v
                             for v in (g.cosths, g.logEs, g.params, g.min_cos_theta)])
    le, af, ab = torch.as_tensor(job.logEs, device=dev), tg(job.aeff_front), tg(job.aeff_back)
    for _ in range(max(3, args.warmup)):
        A.exposure_map(c, w, le, af, ab, ltf)
    torch.cuda.synchronize(dev)
    A.profile_enable(True)
    for _ in range(args.steps):
        A.exposure_map(c, w, le, af, ab, ltf)
    torch.cuda.synchronize(dev)
    prof = A.profile_read()
    A.profile_enable(False)
    n, kms = prof["k_exposure_map_tc"]
    ms = kms / n
    alg = 2 * npix * C * 4 + npix * job.E * 8
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    print(json.dumps({"metric": "exposure-map pixels/s (full sky, tcgen05 3xTF32)", "value": npix / (ms * 1e-3),
                      "unit": "HEALPix pixels/s", "kernel_ms": ms, "launches": n, "nside": nside, "C": C, "E": job.E,
                      "roofline": {"bound": "hbm", "achieved": alg / ms / 1e6, "peak": peak, "unit": "GB/s",
                                   "frac": alg / ms / 1e6 / peak, "alg_bytes_per_launch": alg},
                      "useful_tflops": 2 * npix * 2 * C * job.E * 2 / ms / 1e9}), flush=True)

def spawn_ranks(n: int) -> int:
    """``--gpus N`` without an outer launcher: start N ranks (one process per GPU)
    with torch.distributed.run on 127.0.0.1 and return its exit status.  Fails
    loudly when this machine has fewer than N CUDA devices.  NCCL_DEBUG=INFO makes
    the communicator's rank count visible in the ranks' logs."""
    import socket

    import torch

    have = torch.cuda.device_count() if torch.cuda.is_available() else 0
    if have < n:
        sys.stderr.write(f"bench.py --gpus {n}: this machine has {have} CUDA device(s); "
                         f"one rank per GPU needs {n}\n")
        return 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd, env=env)


def main():
    args = parse()
    if args.exposure_map_nside:
        run_exposure_map(args)
        return
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    rank, world, local_rank = env_rank()
    if args.gpus > 1 and world != args.gpus:
        sys.exit(f"bench.py --gpus {args.gpus} launched with WORLD_SIZE={world}")
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
