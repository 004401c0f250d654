#!/usr/bin/env python
"""Multislice LSQ-ML throughput on B200 (positions x slices per second).

Workload (one "step" = one full LSQ-ML iteration over the scan):
  8 slices of 517x517 (the reference geometry for a 512^2-class field: scan
  span + 2 * (N/2 + 5) px), probe 128x128 with 4 incoherent modes
  (70/15/10/5 %, 25 mrad, 300 kV, 200 A defocus), 64x64 = 4096 positions at
  6 px, mini-batches of 256, amplitude noise model, probe-position
  correction (momentum), patterns at 1e6 e-/pattern -- seeded synthetic
  data with those shapes (no datasets ship here).

  value : pos*slice/s with patterns resident in HBM (device-timed, max over ranks)
  e2e   : the same through the engine API with every step's patterns copied
          from pinned host memory (double-buffered: step k+1's copy runs on a copy
          stream while step k computes; the first copy is inside the timed region)
          and every step's status block read back (while the next step runs)
  roofline : the fused mini-batch kernel (k_group) timed live with CUDA events
          around each launch; algorithmic bytes per pos*slice = N^2 (28 + 16 M) + 4 N^2 / S
  cpu_baseline : the numpy oracle of the same step on the host cores
          (bounded sample: mini-batches of 16 positions at the full shapes).

  --impl reference : times the reference's CPU algorithm (the numpy port in
          oracle/) on this host with all its threads, same metric and config.

Multi-GPU (torchrun): ONE reconstruction split over the ranks (data-parallel:
each mini-batch's positions are divided into contiguous row ranges, the partial
update accumulators are summed with NCCL all-reduces, every rank applies the
same update); value = the reconstruction's pos*slice/s / max rank time
(strong scaling).  --replicas runs independent reconstructions instead (weak
scaling, no collective).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "multislice pos*slice/s (LSQ-ML iteration, 1 B200)"
METRIC_GRAD = "multislice pos*slice/s (gradient-engine iteration, 1 B200)"
UNIT = "pos*slice/s"
CONFIG = {"workload": "multislice LSQ-ML: 8 x 518^2 slices (2 nm), probe 128^2 x 4 modes, "
                      "scan 64x64=4096 @ 6 px, batch 256, position correction on",
          "N": 128, "modes": 4, "slices": 8, "object": [518, 518], "positions": 4096, "batch": 256,
          "solver": "lsqml", "noise_model": "amplitude", "l2": "working set > L2 (1.07 GB psi scratch per batch)"}


def parallelism(world: int, replicas: bool) -> str:
    return f"replicas x{world}" if replicas else ("single GPU" if world == 1 else f"data-parallel x{world}")


def algorithmic_bytes_per_pos_slice(N: int, M: int, S: int, pattern_bytes: int = 4, engine: str = 'lsqml') -> int:
    """O cutout read fwd + adj (16 N^2), psi store + reload (16 M N^2), object-update
    scatter (8 N^2), illumination scatter (4 N^2, LSQ-ML only), pattern read amortised
    over S."""
    illum = 4 if engine == 'lsqml' else 0
    return N * N * (24 + illum + 16 * M) + pattern_bytes * N * N // S


def measured_sm_max_mhz():
    try:
        with open(os.path.join(ROOT, 'MEASURED_PEAKS.json')) as f:
            return float(json.load(f)['sm_max_mhz'])
    except (OSError, KeyError, ValueError):
        return None


def measured_peaks():
    path = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d['hbm_gbs']), 'measured'
    except Exception:
        return 6650.0, 'fallback'


def ncu_traffic_per_launch(engine: str = 'lsqml'):
    """dram bytes (read + write) per k_group launch from the committed ncu summary."""
    path = os.path.join(ROOT, 'profiles', f'k_group_{"grad" if engine == "gradient" else "lsqml"}_c2.md')
    try:
        for line in open(path):
            if line.strip().startswith('traffic_bytes_per_full_launch:'):
                return float(line.split(':', 1)[1].split()[0]) / 1e9   # GB per launch
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(['nvidia-smi', f'--id={self.gpu}', f'--query-gpu={self.Q}',
                                          '--format=csv,noheader,nounits', '-lms', '200'],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for ln in getattr(self, 'lines', []):
            parts = [p.strip() for p in ln.split(',')]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == 'active':
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def setup_dist():
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    return world, rank, local


def cpu_sample(ds, patterns_host, n_groups: int, batch: int, threads: int, seed: int = 5):
    """Time the numpy oracle's LSQ-ML mini-batch step on `n_groups` batches of
    `batch` positions (full shapes).  Returns (pos*slice/s, seconds, description)."""
    from oracle import phaser_np as O
    O.set_fft_workers(threads)
    N = ds.probe.shape[-1]
    S = ds.true_object.shape[0]
    ky, kx = O.recip_grid((N, N), ds.probe_sampling, numpy.float32)
    geom = O.Geometry(numpy.asarray(ds.obj_sampling.corner), numpy.asarray(ds.obj_sampling.sampling), ky, kx,
                      ds.thicknesses)
    props = O.make_propagators(ky, kx, ds.probe_sampling, ds.wavelength, ds.thicknesses)
    rng = numpy.random.default_rng(seed)
    flat = ds.scan.reshape(-1, 2)
    obj = ds.init_object.copy()
    probe = ds.probe.copy()
    # the engine's presolve rescale of the probe intensity (untimed), so the sample runs on the same scale
    idx0 = rng.choice(flat.shape[0], batch, replace=False)
    f = O.epie_dry_run(geom, probe, obj, flat[idx0], patterns_host(idx0), ds.mask, props, None)
    probe = (probe * numpy.sqrt(numpy.mean(f))).astype(probe.dtype)
    t_total = 0.0
    for _ in range(n_groups):
        idx = rng.choice(flat.shape[0], batch, replace=False)
        t0 = time.perf_counter()
        res = O.lsqml_group(geom, probe, obj, flat[idx], patterns_host(idx), ds.mask, props, None,
                            O.NoiseModel(), O.LSQMLParams(), update_position=True)
        t_total += time.perf_counter() - t0
        obj, probe = res['object'], res['probe']
    units = n_groups * batch * S
    return units / t_total, t_total, f"{n_groups} LSQ-ML mini-batches of {batch} positions at the full shapes"


def run_reference(args, world, rank):
    """The reference arm: the CPU (numpy) algorithm timed on this host."""
    if rank != 0:
        return
    from phaser_b200.synthetic import lsqml_multislice_config
    from oracle import phaser_np as O
    threads = os.cpu_count() or 1
    ds = lsqml_multislice_config(seed=0)
    N = ds.probe.shape[-1]
    ky, kx = O.recip_grid((N, N), ds.probe_sampling, numpy.float32)
    geom = O.Geometry(numpy.asarray(ds.obj_sampling.corner), numpy.asarray(ds.obj_sampling.sampling), ky, kx,
                      ds.thicknesses)
    props = O.make_propagators(ky, kx, ds.probe_sampling, ds.wavelength, ds.thicknesses)
    O.set_fft_workers(threads)
    flat = ds.scan.reshape(-1, 2)
    cache = {}

    def pats(idx):   # simulated with the oracle forward model, Poisson at the configured dose
        missing = [int(i) for i in idx if int(i) not in cache]
        if missing:
            psi0, cuts, _, _ = O.cutout_group(geom, ds.probe, ds.true_object, flat[missing])
            psi = O._forward(psi0, cuts, O.tilt_propagators(ky, kx, ds.thicknesses, props, None))
            inten = numpy.sum(O.abs2(O.fft2c(psi[-1] * cuts[:, -1, None])), axis=1)
            inten *= ds.counts / inten.sum(axis=(1, 2), keepdims=True)
            rng = numpy.random.default_rng(1234)
            for i, im in zip(missing, rng.poisson(inten).astype(numpy.float32)):
                cache[i] = im
        return numpy.stack([cache[int(i)] for i in idx])

    batch = args.batch   # the mini-batch size of the GPU arm's line
    S = ds.true_object.shape[0]
    for _ in range(args.warmup):
        cpu_sample(ds, pats, 1, batch, threads, seed=_)
    times = []
    for k in range(args.steps):
        rate, secs, desc = cpu_sample(ds, pats, 1, batch, threads, seed=100 + k)
        times.append(secs)
    t = float(numpy.mean(times))
    value = batch * S / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
            "scaling": "weak" if (args.replicas or world == 1) else "strong",
            "vs_baseline": None, "dtype": "c64", "data": "synthetic", "impl": "reference",
            "config": dict(CONFIG, parallelism=parallelism(world, args.replicas)),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"each step: one LSQ-ML mini-batch of {batch} positions (the line's batch) "
                                       f"at the full shapes (numpy oracle, scipy.fft with {threads} threads; "
                                       f"patterns simulated by the oracle, untimed)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_b200(args, world, rank, local):
    import torch
    import torch.distributed as dist
    from phaser_b200 import _lib
    from phaser_b200.synthetic import lsqml_multislice_config, simulate_patterns
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.engines.gradient import GradientEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL

    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        # NCCL's initialisation log (stderr) shows the ranks and the NVLink / NVLS paths it set up
        os.environ.setdefault('NCCL_DEBUG', 'INFO')
        os.environ.setdefault('NCCL_DEBUG_SUBSYS', 'INIT')
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    lib = _lib.load()

    # CPU baseline first (rank 0, N == 1), before the device is busy.  Data-parallel ranks
    # share one dataset (same seed); replicas each get their own.
    dp = world > 1 and not args.replicas
    ds = lsqml_multislice_config(seed=0 if dp else rank, scan=args.scan)
    pats = simulate_patterns(ds, seed=0 if dp else rank, device=dev)
    config = dict(CONFIG, object=[int(v) for v in ds.obj_sampling.shape])
    if args.scan != 64 or args.batch != 256:   # reduced case (profiling); not the benchmark line
        config.update(workload=f"reduced multislice LSQ-ML (scan {args.scan}x{args.scan}, batch {args.batch})",
                      positions=args.scan * args.scan, batch=args.batch)
    if args.engine == 'gradient':
        config.update(workload=config["workload"].replace("LSQ-ML", "gradient engine (hand-written adjoint, Adam)")
                      .replace(", position correction on", ""), solver="gradient (adam: object 1e-2, probe 1e-3)")
    pats_host = pats.cpu().pin_memory()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        host_np = pats_host.numpy()
        rate, secs, desc = cpu_sample(ds, lambda idx: host_np[idx], 1, args.batch, threads)
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": desc + f" (numpy oracle, scipy.fft with {threads} threads), {secs:.1f} s"}

    N, M, S = ds.probe.shape[-1], ds.probe.shape[0], ds.true_object.shape[0]
    n_pos = int(numpy.prod(ds.scan.shape[:-1]))

    def new_engine(split: bool = False):
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = PL.ConventionalEnginePlan(
            noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
            position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
            niter=10 ** 6, grouping=args.batch, update_positions=True)
        cls = ConventionalEngine
        if split:
            from phaser_b200.distributed import DistributedConventionalEngine as cls
        e = cls({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                 'seed': 'bench', 'recons_name': 'bench'}, props, patterns_on_device=pats)
        e.presolve()
        return e

    def new_gradient_engine():
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = PL.GradientEnginePlan(
            solvers={'object': {'type': 'adam', 'learning_rate': 1e-2}, 'probe': {'type': 'adam', 'learning_rate': 1e-3}},
            noise_model={'type': 'amplitude'}, niter=10 ** 6, grouping=args.batch)
        cls = GradientEngine
        if dp:
            from phaser_b200.distributed import DistributedGradientEngine as cls
        e = cls({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                 'seed': 'bench', 'recons_name': 'bench-grad'}, props, patterns_on_device=pats)
        e.presolve()
        return e

    eng = new_gradient_engine() if args.engine == 'gradient' else new_engine(split=dp)
    stream = torch.cuda.current_stream()
    # FP32 CUDA-core peak of this GPU (FMA probe), the denominator of fp32_pipe.frac
    fp32_measured = None
    if rank == 0:
        tf = ctypes.c_double()
        _lib.call('phb_fp32_peak', 4096, ctypes.byref(tf), None, stream.cuda_stream)
        fp32_measured = tf.value
    it = 0
    for _ in range(args.warmup):
        it += 1
        eng.iteration(it)

    def barrier():
        if world > 1:
            dist.barrier()

    # ---------------- device-resident timing
    eng.fused_events = []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    launches0 = lib.phb_kernel_launches()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            it += 1
            eng.iteration(it, sync=False)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = lib.phb_kernel_launches() - launches0
    eng.check(it)
    barrier()
    t_ms = ev0.elapsed_time(ev1)
    fused = []
    for a, b in eng.fused_events:
        ms = ctypes.c_float()
        _lib.call('phb_event_elapsed_ms', a, b, ctypes.byref(ms))
        fused.append(ms.value)
        _lib.call('phb_event_destroy', a)
        _lib.call('phb_event_destroy', b)
    eng.fused_events = None
    if world > 1:
        tt = torch.tensor([t_ms], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    units_per_step = n_pos * S            # one reconstruction's iteration
    replicas_here = world if not dp else 1   # replicas each run their own reconstruction
    value = replicas_here * units_per_step * args.steps / (t_ms / 1e3)

    # ---------------- end-to-end: host patterns -> device each step, status back each step.
    # Double-buffered: step k+1's patterns are copied from pinned host memory on a copy
    # stream while step k computes; the first step's copy is in the timed region.
    e2e_t = float('nan')
    copy_stream = torch.cuda.Stream(device=dev)
    bufs = [pats, torch.empty_like(pats)]
    copied = [torch.cuda.Event(), torch.cuda.Event()]
    used = [torch.cuda.Event(), torch.cuda.Event()]
    done = [torch.cuda.Event(), torch.cuda.Event()]
    barrier()
    torch.cuda.synchronize()
    if not args.no_e2e:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        bufs[0].copy_(pats_host, non_blocking=True)
        cur = 0
        for k in range(args.steps):
            it += 1
            if k + 1 < args.steps:
                nxt = 1 - cur
                if k > 0:
                    copy_stream.wait_event(used[nxt])   # step k-1 finished reading that buffer
                with torch.cuda.stream(copy_stream):
                    bufs[nxt].copy_(pats_host, non_blocking=True)
                copied[nxt].record(copy_stream)
            eng.eng.set_patterns(bufs[cur])
            eng.iteration(it, sync=False)
            used[cur].record(stream)
            done[k % 2].record(stream)
            if k > 0:   # read the previous step's report while this one runs
                done[(k - 1) % 2].synchronize()
                eng.check(it - 1)
            if k + 1 < args.steps:
                stream.wait_event(copied[1 - cur])
                cur = 1 - cur
        e1.record(stream)
        e1.synchronize()
        eng.check(it)
        e2e_t = e0.elapsed_time(e1) / args.steps
        eng.eng.set_patterns(pats)
    barrier()
    if world > 1:
        tt = torch.tensor([e2e_t], device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_t = float(tt.item())
    e2e_value = replicas_here * units_per_step / (e2e_t / 1e3)
    del bufs

    # ---------------- reconstruction quality: plain LSQ-ML from the flat start, NRMSE vs the true object
    nrmse = None
    if not args.no_nrmse and world == 1:
        nrmse = time_to_target(ds, pats, new_engine, args.nrmse_iters, stream, warm=not args.no_warm)

    extra = None
    if rank == 0 and world == 1 and not args.no_extra:
        extra = extra_configs(dev, stream)

    # ---------------- roofline of the fused kernel
    peak, peak_kind = measured_peaks()
    B = args.batch
    bytes_launch = algorithmic_bytes_per_pos_slice(N, M, S, engine=args.engine) * (B if not dp else -(-B // world)) * S
    avg_ms = float(numpy.mean(fused)) if fused else float('nan')
    achieved = bytes_launch / (avg_ms / 1e3) / 1e9
    traffic = ncu_traffic_per_launch(args.engine)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic if (args.scan == 64 and args.batch == 256) else None,
            "traffic_unit": "GB per launch (ncu)",
            "kernel": ("k_group<128> (fused gradient-engine mini-batch: loss + adjoint)" if args.engine == 'gradient'
                       else "k_group<128> (fused LSQ-ML mini-batch)"),
            "launch": "one mini-batch = the forward launch and the launch resumed at the detector, timed together",
            "launch_ms": avg_ms, "launches_timed": len(fused), "bytes_per_launch": bytes_launch,
            "peak_source": f"{peak_kind} hbm_gbs", "share_of_step": sum(fused) / t_ms if t_ms else None}
    # the kernel's other bound: FP32 FFT work (5 N^2 log2 N^2 per transform, M (4 + 4/S) transforms
    # and ~60 M N^2 elementwise FLOP per position-slice) against the FP32 pipe's peak
    # (148 SMs x 128 FMA lanes x 2 FLOP x max SM clock, an estimate: not in MEASURED_PEAKS.json)
    flop_ps = 5 * N * N * numpy.log2(N * N) * M * (4 + 4 / S) + 60 * M * N * N
    fp32_peak = 148 * 128 * 2 * (measured_sm_max_mhz() or 1965.0) * 1e6
    rows_launch = B if not dp else -(-B // world)   # a data-parallel rank runs its share of the rows
    flops = flop_ps * rows_launch * S / (avg_ms / 1e3)
    roof["fp32_pipe"] = {"achieved_tflops": flops / 1e12, "peak_tflops_estimate": fp32_peak / 1e12,
                         "frac_of_estimate": flops / fp32_peak, "flop_per_pos_slice": flop_ps}
    if fp32_measured:
        roof["fp32_pipe"].update(peak_tflops_measured=fp32_measured, frac=flops / 1e12 / fp32_measured,
                                 peak_source="FMA probe (phb_fp32_peak), measured in this run")

    if rank == 0:
        line = {"metric": METRIC if args.engine == 'lsqml' else METRIC_GRAD, "value": value, "unit": UNIT,
                "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
                "scaling": "strong" if dp else "weak", "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "config": dict(config, parallelism=parallelism(world, args.replicas)),
                "roofline": roof, "cpu_baseline": cpu,
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(pats_host.numel() * 4),
                        "d2h_bytes_per_step": 32},
                "gpu_launches": int(launches), "clocks": clk.summary(), "nrmse": nrmse,
                "other_configs": extra}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def object_nrmse(rec, ref, rows, cols):
    from phaser_b200.metrics import object_nrmse as f
    return f(rec, ref, rows, cols)


def nrmse_race(eng, ref, iters: int, stream, init=None, prep_seconds: float = 0.0, target=None):
    """Run `iters` iterations of `eng` (from `init` when given) and record the NRMSE of
    the projected object after each one against the true object `ref`, with the
    cumulative device time (CUDA events around each iteration) plus prep_seconds."""
    import torch
    from phaser_b200.constraints import RemovePhaseRamp
    crop = RemovePhaseRamp(eng.eng, None, None)
    if init is not None:
        eng.eng.object.copy_(init)
    curve, times = [object_nrmse(eng.eng.object, ref, crop.rows, crop.cols)], [prep_seconds]
    for i in range(1, iters + 1):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.iteration(i, sync=False)
        e1.record(stream)
        e1.synchronize()
        eng.check(i)
        times.append(times[-1] + e0.elapsed_time(e1) / 1e3)
        curve.append(object_nrmse(eng.eng.object, ref, crop.rows, crop.cols))
    out = {"curve": [round(v, 5) for v in curve], "seconds": [round(v, 4) for v in times],
           "prep_seconds": prep_seconds}
    if target is not None:
        hit = next((i for i, v in enumerate(curve) if v <= target), None)
        out.update(iterations_to_target=hit, seconds_to_target=None if hit is None else times[hit])
    return out


ALL_ARMS = ("warm_lsqml", "warm_gradient", "plain_gradient", "warm_gradient_lsqml")


def train_network(geometry: str = 'multislice', slices=(4, 12), seed: int = 7):
    """The warm-start network trained on 196 random-lattice objects x 32^2 positions
    (200,704 patterns) that the forward kernel simulates in `geometry`
    (warmstart.lattice_geometry), 16 epochs of Adam; with its training record."""
    import torch
    from phaser_b200 import warmstart as WS
    spec = WS.DEFAULT_FEATURES
    train_n = 64 if geometry == 'single' else 128
    t0 = time.perf_counter()
    feats, targets = WS.training_set(196, seed=seed, slices=slices, spec=spec, geometry=geometry)
    torch.cuda.synchronize()
    t_data = time.perf_counter() - t0
    fh, th = WS.training_set(4, seed=99, slices=slices, spec=spec, geometry=geometry)
    net = WS.WarmStartNet(seed=0, features=spec, train_n=train_n)
    t0 = time.perf_counter()
    losses = net.train(feats, targets, epochs=16, batch=256, lr=5e-4)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    n_train = int(feats.shape[0])
    del feats, targets
    pred = net.predict(fh)
    info = {
        "description": "3x3 conv encoder/decoder (1-32-64-64-32-2 channels), bf16 weights, fp32 accumulate, "
                       "trained by the library's own kernels on patterns its forward kernel simulated from random "
                       f"lattices (spacing 6-14 px, 0.1-0.5 rad, {slices[0]}-{slices[1]} slices) in the "
                       f"'{geometry}' geometry",
        "training_patterns": n_train, "epochs": 16, "data_seconds": t_data, "training_seconds": t_train,
        "training_loss_per_epoch": [round(v, 5) for v in losses],
        "held_out_patch_mse": float(torch.mean((pred - th) ** 2)), "flat_patch_mse": float(torch.mean(th ** 2))}
    return net, info


def run_c4(args):
    """The learned warm start as the benchmark describes it: the network is trained on
    200,704 patterns that the forward kernel simulates with the single-slice
    configuration's optics (64^2 probe and detector, so the 64x64 input is the whole
    log-scaled pattern; 200 kV, 20 mrad, 100 A defocus, 1 mode, 4 px steps with +-0.5 px
    jitter, 1e5 e-) from random lattices (spacing 6-14 px, 0.1-0.5 rad per slice, 4-12
    slices); its stitched prediction seeds LSQ-ML on a held-out object of that shape
    (drawn from the same generator with another seed); the race records iterations and
    seconds to the plain LSQ-ML run's final NRMSE (`--nrmse-iters` iterations), with the
    residual fallback to the flat start."""
    import torch
    from phaser_b200 import warmstart as WS
    from phaser_b200.synthetic import simulate_patterns
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL
    dev = torch.device('cuda', 0)
    torch.cuda.set_device(dev)
    stream = torch.cuda.current_stream()
    net, info = train_network('single', seed=11)
    ds = next(WS.random_lattice_objects(1, seed=424242, geometry='single'))
    pats = simulate_patterns(ds, seed=77, device=dev, group=64)
    N = ds.probe.shape[-1]

    def new_engine():
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = PL.ConventionalEnginePlan(noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
                                          niter=10 ** 6, grouping=64)
        e = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                                'seed': 'bench-c4', 'recons_name': 'c4'}, props, patterns_on_device=pats)
        e.presolve()
        return e

    res = time_to_target(ds, pats, new_engine, args.nrmse_iters, stream, arms=("warm_lsqml",), net=(net, info))
    print(json.dumps({"metric": "time to the plain LSQ-ML's final NRMSE (s), learned warm start as specified",
                      "config": {"optics": "single-slice configuration: 64^2 probe, 200 kV, 20 mrad, 100 A defocus, "
                                           "1 mode, 32x32 scan @ 4 px +-0.5 px, 1e5 e-",
                                 "held_out_object": f"{ds.true_object.shape[0]} x {ds.true_object.shape[1]}^2 "
                                                    "random lattice", "solver": "LSQ-ML, grouping 64"},
                      "nrmse": res}), flush=True)


def time_to_target(ds, pats, new_engine, iters: int, stream, warm: bool = True, arms=ALL_ARMS, net=None):
    """The benchmark's second metric: device wall time to reach the plain method's final
    object NRMSE.  Arms, all on the benchmark dataset:
      plain_lsqml:   LSQ-ML from the flat object, `iters` iterations; its final NRMSE
                     is the target;
      warm_lsqml:    the same solver from the learned warm start;
      warm_gradient: the gradient engine (hand-written adjoint kernel, Adam on object
                     and probe, amplitude noise model, grouping 256) from the warm start;
      plain_gradient: the gradient engine from the flat object (separates the warm
                     start's share of the gain from the adjoint engine's);
      warm_gradient_lsqml: warm start, 3 gradient-engine iterations, then LSQ-ML
                     polish for the remaining iterations (state handed over on the
                     device; the hand-over time is counted).
    A warm arm's clock starts with the feature extraction, inference, stitching and
    residual tests (prep_seconds).  The network is trained first, once, on 200,704
    simulated patterns; its training time is reported beside, not inside, the race."""
    import torch
    from phaser_b200 import warmstart as WS
    from phaser_b200.engines.gradient import GradientEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL
    ref = torch.from_numpy(ds.true_object).to(pats.device)
    out = {"definition": "projected object (product of slices) over the scanned region, linear phase ramps "
                         "removed, global phase fitted; reference = the true (simulated) object; time = "
                         "device time of the iterations (+ warm-start preparation)"}
    plain = nrmse_race(new_engine(), ref, iters, stream)
    target = plain["curve"][-1]
    # every arm, the plain one included, is timed to the FIRST iteration at which it reaches
    # the target (plain LSQ-ML's NRMSE need not fall monotonically)
    hit = next(i for i, v in enumerate(plain["curve"]) if v <= target)
    plain.update(method="LSQ-ML from the flat start", iterations_to_target=hit, seconds_to_target=plain["seconds"][hit])
    out.update(target_nrmse=target, plain_lsqml=plain)
    if not warm:
        return out
    N = ds.probe.shape[-1]

    # Adam moves every pixel by up to ~learning_rate per mini-batch, so the rates are set
    # per iteration: 1e-2 (object) and 1e-3 (probe) spread over 16 mini-batches (the
    # benchmark's 4096 positions at batch 256), scaled down for more mini-batches
    n_groups = -(-int(numpy.prod(ds.scan.shape[:-1])) // 256)
    lr_scale = min(1.0, 16.0 / n_groups)

    def gradient_engine():
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = PL.GradientEnginePlan(
            solvers={'object': {'type': 'adam', 'learning_rate': 1e-2 * lr_scale},
                     'probe': {'type': 'adam', 'learning_rate': 1e-3 * lr_scale}},
            noise_model={'type': 'amplitude'}, niter=10 ** 6, grouping=256)
        e = GradientEngine({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                            'seed': 'bench', 'recons_name': 'bench-grad'}, props, patterns_on_device=pats)
        e.presolve()
        return e

    net, out["network"] = net if net is not None else train_network()
    # one untimed warm-start pass first: the first launch of each kernel loads its module
    e = new_engine()
    WS.warm_start_object(net, e.eng, pats, ds.scan)
    torch.cuda.synchronize()
    del e
    for arm, make in (("warm_lsqml", new_engine), ("warm_gradient", gradient_engine)):
        if arm not in arms:
            continue
        eng = make()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        init, info = WS.warm_start_object(net, eng.eng, pats, ds.scan)
        torch.cuda.synchronize()
        prep = time.perf_counter() - t0
        r = nrmse_race(eng, ref, iters, stream, init=init, prep_seconds=prep, target=target)
        r["fallback_test"] = info
        out[arm] = r
        del eng
    if "plain_gradient" in arms:
        out["plain_gradient"] = nrmse_race(gradient_engine(), ref, iters, stream, target=target)
    if "warm_gradient_lsqml" in arms:
        chained(out, net, ds, pats, ref, iters, stream, target, new_engine, gradient_engine)
    done = ("plain_lsqml",) + tuple(a for a in ALL_ARMS if a in out)
    out["seconds_to_target"] = {arm: out[arm].get("seconds_to_target") for arm in done}
    out["final_nrmse"] = {arm: out[arm]["curve"][-1] for arm in done}
    # the same race to plain LSQ-ML's BEST NRMSE of the run, and each arm's best
    best = min(plain["curve"])
    to_best = {}
    for arm in done:
        curve, secs = out[arm]["curve"], out[arm]["seconds"]
        i = next((k for k, v in enumerate(curve) if v <= best), None)
        to_best[arm] = None if i is None else secs[i]
    out.update(plain_best_nrmse=best, seconds_to_plain_best=to_best,
               best_nrmse={arm: min(out[arm]["curve"]) for arm in done})
    return out


def chained(out, net, ds, pats, ref, iters, stream, target, new_engine, gradient_engine):
    """Arm warm_gradient_lsqml: warm start, 3 gradient-engine iterations, LSQ-ML polish."""
    import torch
    from phaser_b200 import warmstart as WS
    n_grad = 3
    g = gradient_engine()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    init, info = WS.warm_start_object(net, g.eng, pats, ds.scan)
    torch.cuda.synchronize()
    prep = time.perf_counter() - t0
    first = nrmse_race(g, ref, n_grad, stream, init=init, prep_seconds=prep)
    t0 = time.perf_counter()
    polish = new_engine()
    polish.eng.take_state(g.eng)
    torch.cuda.synchronize()
    handoff = time.perf_counter() - t0
    del g
    second = nrmse_race(polish, ref, iters - n_grad, stream, prep_seconds=first["seconds"][-1] + handoff)
    curve = first["curve"] + second["curve"][1:]
    secs = first["seconds"] + second["seconds"][1:]
    hit = next((i for i, v in enumerate(curve) if v <= target), None)
    out["warm_gradient_lsqml"] = {
        "method": f"warm start, {n_grad} gradient-engine iterations, then LSQ-ML", "curve": curve, "seconds": secs,
        "prep_seconds": prep, "handoff_seconds": handoff, "iterations_to_target": hit,
        "seconds_to_target": None if hit is None else secs[hit], "final_nrmse": curve[-1], "fallback_test": info}
    del polish


def run_large_race(args):
    """Time to the plain LSQ-ML's final NRMSE on the large configuration: plain LSQ-ML
    against warm start -> 3 gradient-engine iterations -> LSQ-ML polish, `--nrmse-iters`
    iterations each.  --spec runs it at the stated size (256^2 probe and detector), else
    with the detector binned 2x2 to 128^2 (see large_multislice_config)."""
    import torch
    from phaser_b200.synthetic import large_multislice_config, simulate_patterns
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL
    dev = torch.device('cuda', 0)
    torch.cuda.set_device(dev)
    ds = large_multislice_config(seed=3, binned=not args.spec)
    pats16 = simulate_patterns(ds, seed=3, device=dev, group=256, counts_u16=True)
    torch.cuda.empty_cache()
    N = ds.probe.shape[-1]

    def new_engine():
        state = ReconsState(iter=IterState(), wavelength=ds.wavelength,
                            probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                            object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                            scan=ds.scan.copy())
        props = PL.ConventionalEnginePlan(
            noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
            position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
            niter=10 ** 6, grouping=256, update_positions=True)
        e = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state, 'dtype': numpy.float32,
                                'seed': 'bench-c5', 'recons_name': 'c5'}, props, patterns_on_device=pats16)
        e.presolve()
        return e

    # the network is trained with this configuration's optics and slice count (28-36 slices)
    net = train_network('large', slices=(28, 36), seed=13)
    res = time_to_target(ds, pats16, new_engine, args.nrmse_iters, torch.cuda.current_stream(),
                         arms=("warm_gradient_lsqml",), net=net)
    size = "256^2 probe and detector (as specified)" if args.spec else "detector binned 2x2 to 128^2"
    print(json.dumps({"metric": f"time to the plain LSQ-ML's final NRMSE (s), large configuration, {size}",
                      "config": {"slices": ds.true_object.shape[0], "object": list(ds.true_object.shape[-2:]),
                                 "N": N, "modes": 8, "positions": int(numpy.prod(ds.scan.shape[:-1])),
                                 "batch": 256, "patterns": "uint16 counts, 5e5 e-, resident"},
                      "nrmse": res}), flush=True)


def large_spec_rate(dev, stream, steps: int = 8, warmup: int = 2, seed: int = 3, scan: int = 256,
                    batch: int = 256):
    """The large configuration as specified (32 x 1033^2 slices, 256^2 probe and detector
    x 8 modes, 65536 positions at 3 px, uint16 counts resident): LSQ-ML and gradient-engine
    throughput over `steps` of the first iteration's mini-batches of `batch` (after
    `warmup`), device time of the group steps (fused launches + update kernels).  A smaller
    `scan` / `batch` is the reduced case of the profiling commands."""
    import torch
    from phaser_b200.synthetic import large_multislice_config, simulate_patterns
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.engines.gradient import GradientEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL
    t0 = time.perf_counter()
    ds = large_multislice_config(seed=seed, scan=scan, binned=False)
    t_obj = time.perf_counter() - t0
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    pats16 = simulate_patterns(ds, seed=seed, device=dev, group=256, counts_u16=True)
    e1.record(stream)
    e1.synchronize()
    t_sim = e0.elapsed_time(e1) / 1e3
    N, S = ds.probe.shape[-1], ds.true_object.shape[0]
    n_pos = int(numpy.prod(ds.scan.shape[:-1]))
    out = {"workload": f"large multislice as specified: {S} x {ds.obj_sampling.shape[0]}^2 slices, probe and "
                       f"detector {N}^2 x 8 modes, {scan}x{scan} scan @ 3 px, 5e5 e-/pattern as uint16 counts resident "
                       f"({pats16.numel() * 2 / 1e9:.1f} GB), batch {batch}",
           "unit": UNIT, "positions": n_pos, "object_setup_seconds": t_obj, "simulation_seconds": t_sim,
           "sample": f"{steps} of the {-(-n_pos // batch)} mini-batches of one iteration, after {warmup}"}

    def state_of():
        return ReconsState(iter=IterState(), wavelength=ds.wavelength,
                           probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                           object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                           scan=ds.scan.copy())

    for kind in ('lsqml', 'gradient'):
        if kind == 'lsqml':
            props = PL.ConventionalEnginePlan(
                noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
                position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
                niter=10 ** 6, grouping=batch, update_positions=True)
            eng = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state_of(), 'dtype': numpy.float32,
                                      'seed': 'bench-c5', 'recons_name': 'c5'}, props, patterns_on_device=pats16)
        else:
            props = PL.GradientEnginePlan(
                solvers={'object': {'type': 'adam', 'learning_rate': 1e-2},
                         'probe': {'type': 'adam', 'learning_rate': 1e-3}},
                noise_model={'type': 'amplitude'}, niter=10 ** 6, grouping=batch)
            eng = GradientEngine({'data': Patterns(None, ds.mask), 'state': state_of(), 'dtype': numpy.float32,
                                  'seed': 'bench-c5', 'recons_name': 'c5-grad'}, props, patterns_on_device=pats16)
        e0.record(stream)
        eng.presolve()
        e1.record(stream)
        e1.synchronize()
        t_pre = e0.elapsed_time(e1) / 1e3
        secs = eng.time_group_steps(1, warmup, steps, stream)
        out[kind] = {"value": steps * batch * S / secs, "ms_per_mini_batch": secs / steps * 1e3,
                     "presolve_seconds": t_pre}
        del eng
        torch.cuda.empty_cache()
    del pats16
    torch.cuda.empty_cache()
    return out


def extra_configs(dev, stream):
    """The other configurations of the benchmark description, measured on the
    same GPU (device time of whole iterations, patterns resident):
      single-slice ePIE: 64^2 probe, 1 mode, 32x32 scan at 4 px (+-0.5 px jitter),
        1e5 e-/pattern, grouping 64, 10 iterations from the flat start;
      gradient engine: 16 x 2 nm slices of 774^2 (reference geometry of a 128x128 scan
        at 5 px), probe 128^2 x 2 modes, Poisson negative log-likelihood, Adam on object
        and probe, grouping 64, 2 timed iterations after 1 warm-up;
      large multislice (detector binned 2x2 to 128^2, see large_multislice_config):
        LSQ-ML and the gradient engine, 1 timed iteration each after 1 warm-up;
      large multislice as specified (256^2 probe and detector): large_spec_rate."""
    import torch
    from phaser_b200.synthetic import (epie_single_slice_config, gradient_multislice_config,
                                       large_multislice_config, simulate_patterns)
    from phaser_b200.engines.conventional import ConventionalEngine
    from phaser_b200.engines.gradient import GradientEngine
    from phaser_b200.state import ReconsState, ProbeState, ObjectState, IterState, Patterns
    from phaser_b200.sampling import Sampling
    from phaser_b200 import plan as PL
    from phaser_b200.constraints import RemovePhaseRamp

    def state_of(ds):
        N = ds.probe.shape[-1]
        return ReconsState(iter=IterState(), wavelength=ds.wavelength,
                           probe=ProbeState(Sampling((N, N), sampling=ds.probe_sampling), ds.probe.copy()),
                           object=ObjectState(ds.obj_sampling, ds.init_object.copy(), ds.thicknesses.copy()),
                           scan=ds.scan.copy())

    def timed(eng, first, n):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for i in range(first, first + n):
            eng.iteration(i, sync=False)
        e1.record(stream)
        e1.synchronize()
        eng.check(first + n - 1)
        return e0.elapsed_time(e1) / 1e3

    out = {}
    ds = epie_single_slice_config(seed=1)
    pats = simulate_patterns(ds, seed=1, device=dev, group=64)
    props = PL.ConventionalEnginePlan(noise_model={'type': 'amplitude'}, solver={'type': 'epie'}, niter=10,
                                      grouping=64)
    eng = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state_of(ds), 'dtype': numpy.float32,
                              'seed': 'bench-c1', 'recons_name': 'c1'}, props, patterns_on_device=pats)
    eng.presolve()
    secs = timed(eng, 1, 10)
    n_pos = int(numpy.prod(ds.scan.shape[:-1]))
    crop = RemovePhaseRamp(eng.eng, None, None)
    ref = torch.from_numpy(ds.true_object).to(dev)
    out['single_slice_epie'] = {
        "workload": "single-slice ePIE: 64^2 probe x 1 mode, 32x32 scan @ 4 px, object "
                    f"{ds.obj_sampling.shape[0]}x{ds.obj_sampling.shape[1]}, grouping 64, 10 iterations",
        "value": n_pos * 1 * 10 / secs, "unit": UNIT, "seconds_10_iterations": secs,
        "nrmse_after_10": object_nrmse(eng.eng.object, ref, crop.rows, crop.cols)}
    del eng, pats
    ds = gradient_multislice_config(seed=2)
    pats = simulate_patterns(ds, seed=2, device=dev, group=256)
    props = PL.GradientEnginePlan(
        solvers={'object': {'type': 'adam', 'learning_rate': 1e-2}, 'probe': {'type': 'adam', 'learning_rate': 1e-3}},
        noise_model={'type': 'poisson', 'eps': 1e-3}, niter=3, grouping=64)
    eng = GradientEngine({'data': Patterns(None, ds.mask), 'state': state_of(ds), 'dtype': numpy.float32,
                          'seed': 'bench-c3', 'recons_name': 'c3'}, props, patterns_on_device=pats)
    eng.presolve()
    timed(eng, 1, 1)
    secs = timed(eng, 2, 2)
    n_pos = int(numpy.prod(ds.scan.shape[:-1]))
    S = ds.true_object.shape[0]
    out['gradient_multislice'] = {
        "workload": f"gradient engine: {S} x {ds.obj_sampling.shape[0]}^2 slices, 128^2 probe x 2 modes, "
                    "128x128 scan @ 5 px, Poisson NLL, Adam, grouping 64",
        "value": n_pos * S * 2 / secs, "unit": UNIT, "ms_per_iteration": secs / 2 * 1e3}
    del eng, pats
    torch.cuda.empty_cache()
    # the large configuration with its 256^2 detector binned to 128^2 (the reference's
    # sim_shape path): 32 x 1033^2 slices, 8 modes, 65536 positions, uint16 counts resident
    ds = large_multislice_config(seed=3)
    pats = simulate_patterns(ds, seed=3, device=dev, group=256)
    peak_count = float(pats.max())
    if peak_count >= 65536:
        raise RuntimeError(f"large configuration: {peak_count} counts do not fit uint16")
    pats16 = pats.to(torch.uint16)
    del pats
    torch.cuda.empty_cache()
    n_pos, S = int(numpy.prod(ds.scan.shape[:-1])), ds.true_object.shape[0]
    large = {"workload": f"large multislice: {S} x {ds.obj_sampling.shape[0]}^2 slices, probe 256^2 x 8 modes with "
                         "the detector binned 2x2 to 128^2 (sim_shape 128, 'resample'), 256x256 scan @ 3 px, "
                         "5e5 e-/pattern as uint16 counts resident (2.1 GB), batch 256",
             "unit": UNIT, "peak_count": peak_count}
    for kind in ('lsqml', 'gradient'):
        if kind == 'lsqml':
            props = PL.ConventionalEnginePlan(
                noise_model={'type': 'amplitude'}, solver={'type': 'lsqml'},
                position_solver={'type': 'momentum', 'step_size': 1e-3, 'max_step_size': 0.2, 'momentum': 0.9},
                niter=10 ** 6, grouping=256, update_positions=True)
            eng = ConventionalEngine({'data': Patterns(None, ds.mask), 'state': state_of(ds), 'dtype': numpy.float32,
                                      'seed': 'bench-c5', 'recons_name': 'c5'}, props, patterns_on_device=pats16)
        else:
            props = PL.GradientEnginePlan(
                solvers={'object': {'type': 'adam', 'learning_rate': 1e-2},
                         'probe': {'type': 'adam', 'learning_rate': 1e-3}},
                noise_model={'type': 'amplitude'}, niter=10 ** 6, grouping=256)
            eng = GradientEngine({'data': Patterns(None, ds.mask), 'state': state_of(ds), 'dtype': numpy.float32,
                                  'seed': 'bench-c5', 'recons_name': 'c5-grad'}, props, patterns_on_device=pats16)
        eng.presolve()
        timed(eng, 1, 1)
        secs = timed(eng, 2, 1)
        large[kind] = {"value": n_pos * S / secs, "seconds_per_iteration": secs}
        del eng
        torch.cuda.empty_cache()
    out['large_multislice_binned'] = large
    del pats16
    torch.cuda.empty_cache()
    # and as specified: 256^2 probe and detector x 8 modes (4-CTA cluster tiles), a sample of
    # 4 mini-batches of 256 after 1 (python bench.py --large-rate times 8 after 2)
    out['large_multislice_spec'] = large_spec_rate(dev, stream, steps=4, warmup=1)
    return out


def run_cnn(args):
    """Throughput of the warm-start network's kernels alone: `args.cnn` random 64x64
    inputs through inference (batch 256) and through training steps (forward,
    backward, Adam; batch 256), CUDA events on the current stream, after warm-up.
    FLOP per pattern: 2 x (multiply-adds of the five 3x3 convolutions) forward,
    3 x that for a training step (forward, data and weight gradients)."""
    import torch
    from phaser_b200 import warmstart as WS
    dev = torch.device('cuda', 0)
    torch.cuda.set_device(dev)
    n = int(args.cnn)
    gen = torch.Generator(device=dev)
    gen.manual_seed(0)
    x = torch.rand((n, 1, 64, 64), generator=gen, device=dev)
    tgt = torch.rand((n, 2, 32, 32), generator=gen, device=dev) * 0.1
    net = WS.WarmStartNet(seed=0)
    macs = 0
    side = 64
    for ci, co, st, relu, up in WS.LAYERS:
        side //= st
        macs += side * side * co * ci * 9
        side *= 2 if up else 1
    flop_fwd = 2 * macs
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    for _ in range(max(1, args.warmup)):
        net.predict(x)
    ev[0].record()
    for _ in range(args.steps):
        net.predict(x)
    ev[1].record()
    net.train(x, tgt, epochs=1, batch=256)
    ev[2].record()
    net.train(x, tgt, epochs=max(1, args.steps // 2), batch=256)
    ev[3].record()
    torch.cuda.synchronize()
    t_inf = ev[0].elapsed_time(ev[1]) / 1e3 / args.steps
    t_train = ev[2].elapsed_time(ev[3]) / 1e3 / max(1, args.steps // 2)
    fp32_peak = 148 * 128 * 2 * (measured_sm_max_mhz() or 1965.0) * 1e6
    print(json.dumps({"metric": "warm-start network patterns/s", "unit": "patterns/s", "patterns": n,
                      "inference": {"value": n / t_inf, "ms": t_inf * 1e3, "tflops": n * flop_fwd / t_inf / 1e12,
                                    "fp32_frac": n * flop_fwd / t_inf / fp32_peak},
                      "training": {"value": n / t_train, "ms_per_epoch": t_train * 1e3,
                                   "tflops": 3 * n * flop_fwd / t_train / 1e12,
                                   "fp32_frac": 3 * n * flop_fwd / t_train / fp32_peak},
                      "flop_per_pattern_forward": flop_fwd}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='b200', choices=['b200', 'reference'])
    ap.add_argument('--replicas', action='store_true',
                    help='N > 1: independent reconstructions per rank (weak scaling) instead of one data-parallel one')
    ap.add_argument('--no-cpu-baseline', action='store_true')
    ap.add_argument('--no-e2e', action='store_true')
    ap.add_argument('--no-nrmse', action='store_true')
    ap.add_argument('--no-extra', action='store_true', help='skip the single-slice ePIE and gradient-engine lines')
    ap.add_argument('--nrmse-iters', type=int, default=20, help='iterations of the NRMSE run (20 = the configuration)')
    ap.add_argument('--no-warm', action='store_true', help='time-to-NRMSE: plain LSQ-ML arm only (no network training)')
    ap.add_argument('--engine', default='lsqml', choices=['lsqml', 'gradient'],
                    help='engine timed for the throughput line (the benchmark configuration is lsqml)')
    ap.add_argument('--scan', type=int, default=64, help='scan side (64 = the benchmark configuration)')
    ap.add_argument('--batch', type=int, default=256, help='mini-batch size (256 = the benchmark configuration)')
    ap.add_argument('--large-race', action='store_true',
                    help='only the time-to-NRMSE race on the large configuration (several minutes)')
    ap.add_argument('--spec', action='store_true',
                    help='--large-race at the stated size (256^2 probe and detector) instead of the binned one')
    ap.add_argument('--c4', action='store_true',
                    help='only the learned warm start as the benchmark describes it (single-slice optics)')
    ap.add_argument('--large-rate', action='store_true',
                    help='only the large configuration at the stated size: LSQ-ML / gradient-engine throughput')
    ap.add_argument('--large-scan', type=int, default=256,
                    help='--large-rate on a smaller square scan (the reduced case of the profiling commands)')
    ap.add_argument('--large-batch', type=int, default=256, help='--large-rate mini-batch size')
    ap.add_argument('--cnn', type=int, default=0, metavar='PATTERNS',
                    help='only time the warm-start network on this many patterns (training step and inference)')
    args = ap.parse_args()
    world, rank, local = setup_dist()
    if args.cnn:
        run_cnn(args)
        return
    if args.large_race:
        run_large_race(args)
        return
    if args.c4:
        run_c4(args)
        return
    if args.large_rate:
        import torch
        dev = torch.device('cuda', 0)
        torch.cuda.set_device(dev)
        print(json.dumps({"metric": "large configuration as specified, pos*slice/s",
                          "large_multislice_spec": large_spec_rate(dev, torch.cuda.current_stream(), args.steps,
                                                                   args.warmup, scan=args.large_scan,
                                                                   batch=args.large_batch)}),
              flush=True)
        return
    if args.impl == 'reference':
        run_reference(args, world, rank)
    else:
        run_b200(args, world, rank, local)


if __name__ == '__main__':
    main()
