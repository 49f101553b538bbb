#!/usr/bin/env python
"""Throughput of the point-source model-map path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c1] [--impl ours|reference]

One step = one pass of the hot path over one batch: exposure -> mean PSF ->
source maps (the three calls of the reference's main.cxx:28-30) for every
source of the workload.  Workload: config c1 (50 point sources, CAR 200x200
@ 0.1 deg, 37 energies 100 MeV - 1 TeV, livetime cube nside 64 x 40), seeded
synthetic inputs.  The metric counts srcmap pixels: one pixel is one
(source, x, y, energy) element of the [S, H, W, E] model map.

For N > 1 (torchrun) every rank runs its own job of the same size (sources are
independent; no collective on the data path): weak scaling, value = all ranks'
pixels / the slowest rank's time.

Prints one JSON line on rank 0.
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

METRIC = "srcmap pixels/sec at 1e-4 rel err (plain GPU cubature path)"
UNIT = "srcmap pixels/s (pixel = one (source, x, y, energy) element)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--config", default="c1")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-graph", action="store_true", help="time eager launches instead of a CUDA graph")
    ap.add_argument("--no-adaptive", action="store_true", help="skip the adaptive-cubature measurement")
    ap.add_argument("--no-surrogate", action="store_true", help="skip training and timing the learned surrogate")
    ap.add_argument("--surrogate-samples", type=int, default=10_000_000)
    ap.add_argument("--surrogate-epochs", type=int, default=20)
    ap.add_argument("--exposure-map-nside", type=int, default=0,
                    help="time only the full-sky exposure map at this nside and exit")
    ap.add_argument("--kernel", default="windows", choices=["windows", "cuda_cores", "tcgen05"],
                    help="FP32 source-map write pass")
    return ap.parse_args()


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


# ----------------------------------------------------------------------------- our arm
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


def run_ours(args, rank, world, local_rank):
    import torch

    from xtsrcmaps_b200 import api as A
    from xtsrcmaps_b200.synth import DESCRIPTIONS, make_job

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    A.init(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)

    # one global source list, CONFIGS[config]["S"] sources per GPU, sharded over
    # the ranks (weak scaling); every rank holds the same livetime cube and IRFs
    from xtsrcmaps_b200.shard import shard_sources
    from xtsrcmaps_b200.synth import CONFIGS

    per_gpu = CONFIGS[args.config]["S"]
    job = make_job(args.config, seed=args.seed, n_sources=per_gpu * world)
    job.src_sph = job.src_sph[shard_sources(job.S, world)[rank]]
    S, H, W, E = job.S, job.wcs.naxis1, job.wcs.naxis2, job.E
    n_values = job.n_values
    # IRF set-up (Irf::collect_irf_data, untimed like the reference's ingest)
    ltf_h = A.livetime_efficiency_factors(job.logEs, job.effic_front)
    nf_h = A.normalize_rpsf(job.rpsf_front, job.scale_front)
    nb_h = A.normalize_rpsf(job.rpsf_back, job.scale_back)
    d = to_device_job(job, torch, dev)
    from xtsrcmaps_b200.irf import IrfGrid

    tt = lambda a: torch.as_tensor(np.asarray(a), device=dev, dtype=torch.float64)
    nf = IrfGrid(tt(nf_h.cosths), tt(nf_h.logEs), tt(nf_h.params), nf_h.min_cos_theta)
    nb = IrfGrid(tt(nb_h.cosths), tt(nb_h.logEs), tt(nb_h.params), nb_h.min_cos_theta)
    ltf = tt(ltf_h)
    out = torch.empty((S, H, W, E), dtype=torch.float32, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    stream = torch.cuda.Stream(dev)

    # one step = the public call that replaces main.cxx:28-30 (point_source_maps:
    # exposure, mean PSF and model maps; the map geometry runs on a second stream
    # beside exposure and PSF); step3 = the three separate calls, for comparison
    def step():
        with torch.cuda.stream(stream):
            A.point_source_maps(job.wcs, d["src"], d["cube"], d["wcube"], d["logEs"], d["af"], d["ab"], nf, nb,
                                ltf, out=out, with_info=False, kernel=args.kernel)

    def step3():
        with torch.cuda.stream(stream):
            ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
            A.point_src_model_map_wcs(job.wcs, d["src"], ex.exposure, ps.uPsf, ps.partial_psf_integral, kernel=args.kernel,
                                      out=out, with_info=False)

    for _ in range(max(3, args.warmup)):
        step3()
        step()
    torch.cuda.synchronize(dev)

    # One step captured into a CUDA graph: once warm, the library's device-pointer
    # calls neither allocate nor synchronise, so the three calls replay as one
    # launch.  Two graphs: a plain one for the timed steps, and one whose kernels
    # are bracketed by the library's timers (event-record nodes) for the per-kernel
    # table and the roofline, replayed over the same number of steps afterwards.
    def capture(profiled, fn=step):
        A.profile_enable(True, keep=True) if profiled else A.profile_enable(False)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            fn()
        for _ in range(max(3, args.warmup)):
            with torch.cuda.stream(stream):
                g.replay()
        torch.cuda.synchronize(dev)
        if profiled:
            A.profile_read()
        return g

    graph = gprof = graph3 = None
    graph_note = "eager launches"
    if not args.no_graph:
        try:
            graph = capture(False)
            graph3 = capture(False, step3)
            gprof = capture(True)  # last: enabling or disabling the profiler clears its records
            graph_note = "one CUDA graph per step (the fused public call captured once)"
        except Exception as exc:  # capture refused: time eager launches
            graph = gprof = graph3 = None
            graph_note = "eager launches (graph capture failed: %s)" % str(exc).splitlines()[0][:120]
            A.profile_enable(False)
            torch.cuda.synchronize(dev)

    def timed(run, per_step=None):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        torch.cuda.synchronize(dev)
        if dist:
            dist.barrier()
        for k in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()  # L2 flush between timed steps (outside the events)
            evs[k][0].record(stream)
            run()
            evs[k][1].record(stream)
            if per_step:
                stream.synchronize()
                per_step()
        torch.cuda.synchronize(dev)
        return sum(a.elapsed_time(b) for a, b in evs)

    def replay(g):
        def run():
            with torch.cuda.stream(stream):
                g.replay()
        return run

    prof = {}

    def add_prof(p):
        for k_, (n_, ms_) in p.items():
            a_ = prof.get(k_, (0, 0.0))
            prof[k_] = (a_[0] + n_, a_[1] + ms_)

    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    t0 = time.time()
    if graph is not None:
        ms = timed(replay(graph))
        t1 = time.time()
        # per-kernel times: the instrumented graph (its timers were recorded at
        # capture and are kept), read after every replay
        ms_prof = timed(replay(gprof), lambda: add_prof(A.profile_read()))
        ms3 = timed(replay(graph3))
    else:
        A.profile_enable(True)
        ms = timed(step)
        t1 = time.time()
        add_prof(A.profile_read())
        ms_prof = ms
        A.profile_enable(False)
        ms3 = timed(step3)
    A.profile_enable(False)
    ck = clocks.stop(t0, t1)

    # the same pipeline with adaptive Genz-Malik cubature of each pixel in place
    # of the 12-point rule (rtol 1e-4, depth 6), eager launches, same timing rules
    adaptive = None
    if not args.no_adaptive:
        out_a = torch.empty_like(out)  # its own buffer: `out` keeps the 12-point map for the error check
        def step_adaptive():
            with torch.cuda.stream(stream):
                ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
                ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
                A.point_src_model_map_wcs_adaptive(job.wcs, d["src"], ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                                   rtol=1e-4, max_depth=6, out=out_a, with_info=False)

        for _ in range(max(3, args.warmup)):
            step_adaptive()
        ka = max(3, min(args.steps, 10))
        ea = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ka)]
        torch.cuda.synchronize(dev)
        for k in range(ka):
            with torch.cuda.stream(stream):
                flush.zero_()
            ea[k][0].record(stream)
            step_adaptive()
            ea[k][1].record(stream)
        torch.cuda.synchronize(dev)
        ms_a = sum(a_.elapsed_time(b_) for a_, b_ in ea) / ka
        adaptive = {"value": n_values * world / (ms_a * 1e-3), "unit": UNIT, "ms_per_step": ms_a, "steps": ka,
                    "rtol": 1e-4, "max_depth": 6,
                    "note": "point_src_model_map_wcs_adaptive (Genz-Malik 7/5 per pixel) in place of the 12-point "
                            "rule; eager launches; accuracy vs the converged pixel integral is in the tests"}
    # the autotuner's write-pass choice on this job (each kernel timed on the job's own geometry)
    from xtsrcmaps_b200.autotune import tune_write_pass

    with torch.cuda.stream(stream):
        ex_t = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
        ps_t = A.compute_psf_data(nf, nb, ex_t, d["logEs"], ltf)
        autotune = tune_write_pass(job.wcs, d["src"], ex_t.exposure, ps_t.uPsf, ps_t.partial_psf_integral)
    surrogate = None
    if not args.no_surrogate:
        surrogate = bench_surrogate(args, A, job, d, nf, nb, ltf, out, flush, stream, dev, n_values, world)
    ms_t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if dist:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms_max = float(ms_t.item())
    value = n_values * world * args.steps / (ms_max * 1e-3)

    # roofline of the write pass (k_srcmap, the kernel that writes the srcmap values), measured
    # inside the timed region
    kname = "k_srcmap"
    launches, kms = prof.get(kname, (0, 0.0))
    epad = (E + 3) // 4 * 4
    alg_bytes = 4 * n_values + 4 * S * 401 * epad + 24 * (H + 1) * (W + 1) + 8 * H * W
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    # the write pass runs once per chunk of sources; its algorithmic bytes per launch are
    # the step's bytes divided by the launches per step
    per_step = launches / args.steps if launches else 1
    alg_bytes = alg_bytes / per_step
    achieved = alg_bytes / (kms / launches * 1e-3) / 1e9 if launches else None
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "k_srcmap_c1_traffic.json")))
        if tr.get("workload") == args.config and args.kernel == "windows":
            traffic = tr.get("dram_bytes_per_launch")
    except (OSError, ValueError):
        pass
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None, "peak_source": peak_src,
                "traffic": traffic, "alg_bytes_per_launch": int(alg_bytes), "launches_per_step": per_step,
                "avg_launch_ms": kms / launches if launches else None,
                "kernel_share": kms / ms_prof if ms_prof else None,
                "kernel_timing": "library CUDA events around each kernel, from %d instrumented steps "
                                 "(%.4f ms/step with the timers)" % (args.steps, ms_prof / args.steps)}
    kernels = {k: {"launches": v[0], "ms": round(v[1], 4)} for k, v in prof.items()}
    # the kernel with the largest share of the instrumented step, and the path as a whole
    # against HBM (4 B written per value)
    dom = max(prof.items(), key=lambda kv: kv[1][1]) if prof else None
    dominant = None
    if dom:
        dominant = {"kernel": dom[0], "share": dom[1][1] / ms_prof if ms_prof else None,
                    "avg_launch_ms": dom[1][1] / dom[1][0] if dom[1][0] else None}
        if dom[0] == "k_pixel_windows":
            dominant["bound"] = ("FP64 issue and shared-memory latency (geometry of 12 points per pixel; "
                                 "~2 % of DRAM bandwidth): not an HBM or tensor kernel")
    path_gbs = 4.0 * n_values * world / (ms_max / args.steps * 1e-3) / 1e9
    roofline_path = {"bound": "hbm", "achieved": path_gbs, "peak": peak, "unit": "GB/s", "frac": path_gbs / peak,
                     "note": "whole step: 4 B written per srcmap value over the step time"}
    gpu_launches = sum(v[0] for v in prof.values())

    # end to end through the public API with host (pinned) buffers: the fused
    # call that replaces main.cxx:28-30, and the three separate calls
    e2e = None
    if not args.no_e2e:
        hp = pinned_job(job, torch)
        hout = torch.empty((S, H, W, E), dtype=torch.float32).pin_memory().numpy()

        def step_fused():
            A.point_source_maps(job.wcs, hp["src"], hp["cube"], hp["wcube"], hp["logEs"], job.aeff_front,
                                job.aeff_back, nf_h, nb_h, ltf_h, out=hout, with_info=False, kernel=args.kernel)

        def step_three():
            ex = A.compute_exposure(hp["cube"], hp["wcube"], hp["logEs"], hp["src"], job.aeff_front,
                                    job.aeff_back, ltf_h)
            ps = A.compute_psf_data(nf_h, nb_h, ex, hp["logEs"], ltf_h)
            A.point_src_model_map_wcs(job.wcs, hp["src"], ex.exposure, ps.uPsf, ps.partial_psf_integral,
                                      kernel=args.kernel, out=hout, with_info=False)

        ke = max(3, min(args.steps, 20))

        def wall(fn):
            for _ in range(3):
                fn()
            if dist:
                dist.barrier()
            t0_ = time.perf_counter()
            for _ in range(ke):
                fn()
            te_ = time.perf_counter() - t0_
            te_t = torch.tensor([te_], dtype=torch.float64, device=dev)
            if dist:
                dist.all_reduce(te_t, op=dist.ReduceOp.MAX)
            return float(te_t.item())

        te = wall(step_fused)
        te3 = wall(step_three)
        C = int(job.exp_cube.nbrbins)
        grid_b = lambda g: 8 * (g.cosths.size + g.logEs.size + g.params.size)
        # with host buffers the library uploads only the livetime rows at the sources' pixels
        # (their indices come back first, 8 B per source)
        cube_b = 2 * 4 * S * C
        h2d = (cube_b + 8 * E + 8 * 2 * S + grid_b(job.aeff_front) + grid_b(job.aeff_back)
               + grid_b(nf_h) + grid_b(nb_h) + 8 * 2 * E)
        d2h = 4 * n_values + 8 * S
        h2d3 = (cube_b + 8 * E + 8 * 2 * S + grid_b(job.aeff_front) + grid_b(job.aeff_back)
                + 8 * 2 * E  # exposure
                + grid_b(nf_h) + grid_b(nb_h) + 8 * (C + E + 2 * C * E + 2 * S * C + 2 * E + S * E)  # psf
                + 8 * (2 * S + S * E + 2 * S * 401 * E))  # srcmap
        d2h3 = (8 * S + 8 * (C + 2 * C * E + 2 * S * C + S * E) + 8 * 2 * S * 401 * E + 4 * n_values)
        e2e = {"value": n_values * world * ke / te, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": ke,
               "note": "one public call per step (point_source_maps: the three calls of main.cxx:28-30 fused) "
                       "from pinned host buffers to a pinned host map, copies inside the timed region",
               "three_calls": {"value": n_values * world * ke / te3, "h2d_bytes_per_step": int(h2d3),
                               "d2h_bytes_per_step": int(d2h3),
                               "note": "compute_exposure, compute_psf_data, point_src_model_map_wcs as "
                                       "separate host-buffer calls"}}

    cpu = None
    err = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, err = cpu_baseline(job, out.cpu().numpy())

    graph = gprof = None  # release the captured graphs before the process group goes away
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": max(3, args.warmup), "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (separations, sums and tables f64)",
        "data": "synthetic (seeded livetime cube, IRF tables and source positions; no public dataset)",
        "config": {"workload": args.config + ": " + DESCRIPTIONS[args.config], "sources_per_gpu": S,
                   "map": f"{H}x{W}", "energies": E, "values_per_step_per_gpu": n_values,
                   "parallelism": f"sources sharded over {world} GPU(s), no data-path collective",
                   "l2": "256 MiB buffer written between timed steps (L2 flush); the 296 MB map "
                         "written per step also exceeds the 126 MB L2",
                   "output_dtype": "float32", "launch": graph_note},
        "roofline": roofline, "dominant_kernel": dominant, "roofline_path": roofline_path,
        "kernels": kernels, "gpu_launches": gpu_launches,
        "clocks": ck, "e2e": e2e, "cpu_baseline": cpu, "max_rel_err_vs_fp64_oracle": err,
        "adaptive": adaptive, "surrogate": surrogate, "autotune_write_pass": autotune,
        "three_calls_device": {"ms_per_step": ms3 / args.steps, "value": n_values * world * args.steps / (ms3 * 1e-3),
                               "note": "compute_exposure, compute_psf_data, point_src_model_map_wcs as three "
                                       "device-pointer calls on one stream (no geometry overlap)"},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- surrogate
def bench_surrogate(args, A, job, d, nf, nb, ltf, out, flush, stream, dev, n_values, world):
    """The learned surrogate on the bench job: trained on the GPU (untimed) on
    samples of the 12-point rule around the mean PSFs of a 500-source job of
    another seed, its error on fresh samples of a third seed against the centre
    value alone, then the same step as the plain path (exposure, mean PSF, model
    map) with the surrogate's model map, timed with the same rules."""
    import numpy as np
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
    hj, hu = tables(args.seed + 200)
    Xh, Yh = samples(hu, hj.logEs, 1_000_000, seed=args.seed + 2)
    yp = net.predict(Xh)
    rho2 = (10.0 ** Xh[:, 0].double()) ** 2
    err_net = ((yp.double() - Yh.double()).abs() / rho2)
    err_c = Yh.double().abs() / rho2
    held = {"samples": int(Xh.shape[0]), "rms_rel_err": float(err_net.pow(2).mean().sqrt()),
            "max_rel_err": float(err_net.max()), "frac_within_1e-4": float((err_net <= 1e-4).double().mean()),
            "centre_value_rms_rel_err": float(err_c.pow(2).mean().sqrt()),
            "centre_value_max_rel_err": float(err_c.max())}
    held["gain_rms"] = held["centre_value_rms_rel_err"] / held["rms_rel_err"]
    del Xh, Yh, yp
    out_s = torch.empty_like(out)
    stats = {}

    def step_sur():
        with torch.cuda.stream(stream):
            ex = A.compute_exposure(d["cube"], d["wcube"], d["logEs"], d["src"], d["af"], d["ab"], ltf)
            ps = A.compute_psf_data(nf, nb, ex, d["logEs"], ltf)
            m, _, st = A.point_src_model_map_wcs_surrogate(job.wcs, d["src"], ex.exposure, ps.uPsf,
                                                           ps.partial_psf_integral, d["logEs"], net,
                                                           check_tol=1e-4, with_info=False)
            out_s.copy_(m)
            stats.update(st)

    for _ in range(max(3, args.warmup)):
        step_sur()
    ks = max(3, min(args.steps, 5))
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(ks)]
    torch.cuda.synchronize(dev)
    for k in range(ks):
        with torch.cuda.stream(stream):
            flush.zero_()
        ev[k][0].record(stream)
        step_sur()
        ev[k][1].record(stream)
    torch.cuda.synchronize(dev)
    ms_s = sum(a_.elapsed_time(b_) for a_, b_ in ev) / ks
    A.profile_enable(True)
    step_sur()
    prof = A.profile_read()
    A.profile_enable(False)
    rel = ((out_s.double() - out.double()).abs() / out.double().abs().clamp_min(1e-300))
    fwd_ms = prof.get("k_mlp_forward", (0, 0.0))[1]
    rows = int(stats.get("evaluated", n_values))  # the network runs only on the values it may take
    flop = 2 * (5 * 128 + 2 * 128 * 128 + 128) * rows
    return {"value": n_values * world / (ms_s * 1e-3), "unit": UNIT, "ms_per_step": ms_s, "steps": ks,
            "check_tol": 1e-4, "rho_min": net.rho_min, "stats": stats,
            "accepted_frac": stats.get("accepted", 0) / max(1, stats.get("values", 1)),
            "max_rel_err_vs_plain_map": float(rel.max()), "frac_within_1e-4_vs_plain_map": float((rel <= 1e-4).double().mean()),
            "network_forward": {"ms": fwd_ms, "rows": rows, "tflops": flop / (fwd_ms * 1e-3) / 1e12 if fwd_ms else None,
                                "note": "67,072 FLOP per row (5-128-128-128-1); the two hidden layers on tcgen05"},
            "train": {"samples": args.surrogate_samples, "epochs": args.surrogate_epochs, "seconds": t_train,
                      "first_epoch_loss": losses[0], "final_loss": losses[-1],
                      "psf_tables": "c2-style job (500 sources) of another seed"},
            "held_out": held,
            "note": "pixel means from the network where the centre is >= rho_min pixel sizes from the source and "
                    "the features lie in the training range, the FP64 12-point rule elsewhere; every 61st pixel "
                    "checked against the rule and a map whose check exceeds check_tol redone by the rule; "
                    "step = exposure + mean PSF + surrogate model map, eager launches"}


# ----------------------------------------------------------------------------- CPU legs
def _oracle_worker(args):
    name, seed, lo, hi = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import oracle_pipeline
    from xtsrcmaps_b200.synth import make_job

    job = make_job(name, seed=seed)
    job.src_sph = job.src_sph[lo:hi]
    t0 = time.perf_counter()
    r = oracle_pipeline(job)
    return time.perf_counter() - t0, r["map"].size


def _reference_runner(job):
    """One full pass of the CPU reference over ``job``: the reference's own code
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
            f"the {job.S} sources of the cubature")
    return (lambda: reference_pipeline(job, setup)), threads, desc


def cpu_baseline(job, gpu_map):
    """The CPU reference (compiled reference code, else the FP64 oracle port) on
    the host cores over the bench's own job, repeated for about 10 s; also the
    GPU map's error against the FP64 oracle."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from helpers import max_rel, oracle_pipeline

    r = oracle_pipeline(job)
    err = max_rel(gpu_map, r["map"])
    run, threads, desc = _reference_runner(job)
    kind = "reference"
    if run is None:
        run, threads, kind = (lambda: oracle_pipeline(job)), 1, "port"
        desc = "the FP64 oracle (a scalar C restatement of the reference path) on one core"
    run()
    t0 = time.perf_counter()
    reps = 0
    while reps < 1 or (time.perf_counter() - t0 < 10.0 and reps < 20):
        run()
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return ({"value": job.n_values / dt, "unit": UNIT, "cores": threads, "kind": kind,
             "sample": f"the full bench job ({job.S} sources, {job.wcs.naxis1}x{job.wcs.naxis2}, {job.E} "
                       f"energies) {reps} times: {desc}"}, err)


def run_reference(args, rank, world):
    """--impl reference: the CPU reference on this box's host cores (rank 0 only)."""
    if rank != 0:
        return
    from xtsrcmaps_b200.synth import DESCRIPTIONS, make_job

    job = make_job(args.config, seed=args.seed)
    run, threads, desc = _reference_runner(job)
    if run is not None:
        kind = "reference"
        warm = 0
        t_w = time.perf_counter()
        while warm < max(3, args.warmup) and (warm < 3 or time.perf_counter() - t_w < 30.0):
            run()
            warm += 1
        times = []
        t_all = time.perf_counter()
        for _ in range(args.steps):  # each step is the whole workload; stop after ~60 s
            t0 = time.perf_counter()
            run()
            times.append(time.perf_counter() - t0)
            if time.perf_counter() - t_all > 60.0:
                break
        sample = f"the whole {args.config} job per step: {desc}"
    else:  # the oracle port, one process per block of sources
        import multiprocessing as mp

        kind = "port"
        cores = os.cpu_count() or 1
        S = job.S
        chunks = [(args.config, args.seed, i * S // cores, (i + 1) * S // cores) for i in range(cores)]
        chunks = [c for c in chunks if c[3] > c[2]]
        threads = len(chunks)
        ctx = mp.get_context("spawn")
        with ctx.Pool(len(chunks)) as pool:
            warm = max(3, min(args.warmup, 5))
            for _ in range(warm):
                pool.map(_oracle_worker, chunks)
            times = []
            for _ in range(max(1, min(args.steps, 5))):
                t0 = time.perf_counter()
                pool.map(_oracle_worker, chunks)
                times.append(time.perf_counter() - t0)
        sample = f"the whole {args.config} job per step, FP64 oracle split by source over {threads} processes"
    ms = 1e3 * sum(times) / len(times)
    value = job.n_values / (ms * 1e-3)
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


def main():
    args = parse()
    if args.exposure_map_nside:
        run_exposure_map(args)
        return
    rank, world, local_rank = env_rank()
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
