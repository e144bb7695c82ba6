"""Benchmark of the batched SSFM sweep on B200 (one JSON line on rank 0).

Workload: the batched parameter sweep — 256 instances from seed 0 with grid side in
{64, 128, 192, 256}, nz in [100, 400], P log-uniform 1-50 W, w0 15-60 µm, focus anywhere
in the crystal, oven 20-80 °C, L in {10, 20} mm — run in FP32 through the fused
persistent march (one launch per grid-size class, classes on concurrent streams).  One
step = one whole sweep: every instance marches its nz-1 SSFM steps.  Metric: grid-point
steps per second, sum over instances of N^2 (nz-1) divided by the time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision 32|64] [--impl ours|reference]

Under torchrun every rank runs its own sweep (seed = rank): weak scaling, no collective
on the data path; the time is the max over ranks.  `--scaling strong` instead splits one
sweep over the ranks (cushg_b200/shard.py, greedy by cost).  `--impl reference` times the CPU
restatement of the reference (oracle/, FP32 like the reference) on the host cores over a
bounded sample of the same sweep; rank 0 only.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from cushg_b200 import params as P  # noqa: E402

B200_SMS = 148
FP32_LANES_PER_SM = 128
# DRAM bytes (read + write) per launch of the dominant kernel of the sweep, the 256 x 256 FP32
# class (ssfm_plain_kernel<float, 256, 16, 256>), from one ncu launch-list capture of this
# bench (`--steps 2 --warmup 3 --no-cpu-baseline --no-autotune --no-extras`, dram__bytes_read.sum
# and dram__bytes_write.sum); the fields stay on chip, so this is descriptors and outputs
SWEEP_256_DRAM_BYTES_PER_LAUNCH = 9.78e6
# bytes of one instance descriptor the batch call uploads (shg::InstDesc)
INST_DESC_BYTES = 376


def flops_per_point_step(n: int) -> float:
    """Algorithmic flops of one SSFM step per grid point (counted in real flops, FMA = 2):
    four 2D FFTs of n x n at 5 log2(n^2) each (2 fields, forward + inverse), the two
    propagator products (6 each) and two applications of the reference's RK4 scheme at
    192 flops each (4 evaluations of dA/dz at 35, 3 stage inputs at 8, the weighted sum
    at 20 and the update at 8)."""
    return 4 * 5 * math.log2(n * n) + 2 * 6 + 2 * 192


def point_steps(ps) -> int:
    return int(sum(p.nx * p.ny * (p.nz - 1) for p in ps))


def algorithmic_flops(ps) -> float:
    return float(sum(p.nx * p.ny * (p.nz - 1) * flops_per_point_step(p.nx) for p in ps))


def workload_params(args, rank: int):
    """The sweep (default) or, with --class-side, `--class-count` copies of one grid-size class
    (a small case for profiling one kernel variant)."""
    if args.class_side:
        base = P.config_sweep(256, seed=rank, precision=args.precision)
        pick = [p for p in base if p.nx == args.class_side] or [P.workload(args.class_side, 100, 20000.0, 20.0, 30.0,
                                                                             10000.0, 40.0, precision=args.precision)]
        return [pick[i % len(pick)].replace(nz=args.class_nz) for i in range(args.class_count)]
    return P.config_sweep(256, seed=rank, precision=args.precision)


def sample_stride(ps, count: int):
    step = max(1, len(ps) // count)
    return ps[::step][:count]


# ---------------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        rows = []
        if self.path and os.path.exists(self.path):
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    try:
                        rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
                    except ValueError:
                        pass
            os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------- our solver
def run_ours(args, rank: int, world: int, local_rank: int) -> dict | None:
    import torch
    from cushg_b200 import shg

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    ps = workload_params(args, rank)
    total_pts = world * point_steps(ps)
    if args.scaling == "strong" and not args.class_side:
        # one sweep (seed 0) split across the ranks, greedy by cost; no data-path collective
        from cushg_b200 import shard
        full = P.config_sweep(256, seed=0, precision=args.precision)
        _, ps = shard.shard(full, rank, world)
        total_pts = point_steps(full)
    if args.precision == 32 and args.fp32_guard > 0:
        # instances whose predicted FP32 SH field error exceeds the guard run the FP64 march
        ps = [p.replace(fp32_guard=args.fp32_guard) for p in ps]
    cdt = torch.complex64 if args.precision == 32 else torch.complex128
    pumps = [torch.empty((p.ny, p.nx), dtype=cdt, device=dev) for p in ps]
    sigs = [torch.empty((p.ny, p.nx), dtype=cdt, device=dev) for p in ps]
    stream = torch.cuda.current_stream(dev)
    sptr = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)  # > 126 MB L2

    # the launch schedule of each grid-size class, chosen on this device by the time of this
    # whole batch (untimed): the classes share the SMs, so a class's fastest split alone can
    # slow the sweep
    tuned = []
    if args.class_side and args.class_schedule:
        c, t = (int(v) for v in args.class_schedule.split(","))
        shg.set_schedule(args.precision, args.class_side, c, t)
        tuned.append({"n": args.class_side, "cluster": c, "threads": t, "candidates": 1, "gain": 1.0})
    elif not args.no_autotune:
        for r in shg.autotune_batch(ps):
            tuned.append({"n": r["n"], "cluster": r["cluster"], "threads": r["threads"], "candidates": r["candidates"],
                          "gain": r["pt_steps_per_s"] / r["default_pt_steps_per_s"]})

    def sweep():
        shg.solve_batch_device(ps, pumps, sigs, stream=sptr, want_power=False)

    for _ in range(args.warmup):
        sweep()
    torch.cuda.synchronize()

    # device-timed region: inputs (descriptors) already resident after warm-up... the
    # descriptor upload is part of every call; the fields never leave the chip
    # each step starts from an idle device after an L2 flush, like the end-to-end calls below,
    # and both take the median over their steps
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            evs[k][0].record(stream)
            sweep()
            evs[k][1].record(stream)
            torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    times = [a.elapsed_time(b) for a, b in evs]
    ms = statistics.median(times)

    # end to end through the C ABI with host buffers (shg_solve_batch): parameter sets in,
    # SH powers and both output fields back into pinned host memory every step, each
    # grid-size class's fields copied as soon as its march ends
    host_p = [torch.empty((p.ny, p.nx), dtype=cdt, pin_memory=True) for p in ps]
    host_s = [torch.empty((p.ny, p.nx), dtype=cdt, pin_memory=True) for p in ps]
    shg.solve_batch(ps, host_p, host_s)  # untimed: the call's own set-up
    e2e_t = []
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        shg.solve_batch(ps, host_p, host_s)
        e2e_t.append(time.perf_counter() - t0)
    e2e_ms = 1e3 * statistics.median(e2e_t)
    d2h = sum(2 * p.nx * p.ny * (8 if args.precision == 32 else 16) for p in ps) + 16 * len(ps)
    h2d = len(ps) * INST_DESC_BYTES

    # the dominant kernel alone: the largest grid-size class as one launch on this stream,
    # timed with CUDA events (the sweep runs the classes concurrently on forked streams)
    nmax = max(p.nx for p in ps)
    # the FP32 instances of the largest class (instances a guard promotes run another kernel)
    dom_i = [i for i, p in enumerate(ps)
             if p.nx == nmax and not (p.fp32_guard > 0 and shg.fp32_error_estimate(p) > p.fp32_guard)]
    dom = [ps[i] for i in dom_i]
    dom_ms = []
    for k in range(args.steps):
        flush.fill_(k & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        shg.solve_batch_device(dom, [pumps[i] for i in dom_i], [sigs[i] for i in dom_i], stream=sptr,
                               want_power=False)
        b.record(stream)
        torch.cuda.synchronize()
        dom_ms.append(a.elapsed_time(b))
    dom_ms = statistics.median(dom_ms)

    if dist is not None:
        t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms, e2e_ms = float(t[0]), float(t[1])
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None

    pts = point_steps(ps)
    value = total_pts / (ms * 1e-3)
    e2e_value = total_pts / (e2e_ms * 1e-3)
    clocks = clk.summary()

    # roofline of the fused march, FP32 (or FP64) CUDA-core issue bound: the dominant kernel
    # (largest class) alone, and the whole sweep
    fl = algorithmic_flops(ps)
    sweep_tflops = fl / (ms * 1e-3) / 1e12
    achieved_tflops = algorithmic_flops(dom) / (dom_ms * 1e-3) / 1e12
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    lanes = FP32_LANES_PER_SM if args.precision == 32 else FP32_LANES_PER_SM // 2
    peak = B200_SMS * lanes * 2 * sm_mhz * 1e6 / 1e12
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    alg_bytes = pts * (32 if args.precision == 32 else 64)
    hbm_achieved = alg_bytes / (ms * 1e-3) / 1e9

    # accuracy of this precision against the FP64 path on the same sweep
    err = None
    if args.precision == 32 and not args.class_side:
        ps64 = [p.replace(precision=64, fp32_guard=0.0) for p in ps]
        p32 = shg.solve_batch_device(ps, None, None, stream=sptr)
        p64 = shg.solve_batch_device(ps64, None, None, stream=sptr)
        rel = np.abs(p32 - p64) / np.abs(p64)
        err = {"sh_power_rel_max": float(rel.max()), "sh_power_rel_median": float(np.median(rel))}

    # the same sweep with every instance in FP32 (no guard): its rate and its error, beside the
    # guarded headline (same schedules, timing as above, fewer steps)
    unguarded = None
    if args.precision == 32 and args.fp32_guard > 0 and not args.class_side and not args.no_extras:
        pu = [p.replace(fp32_guard=0.0) for p in ps]
        for _ in range(2):
            shg.solve_batch_device(pu, pumps, sigs, stream=sptr, want_power=False)
        tu = []
        for k in range(max(3, args.steps // 2)):
            flush.fill_(k & 0xFF)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            shg.solve_batch_device(pu, pumps, sigs, stream=sptr, want_power=False)
            b.record(stream)
            torch.cuda.synchronize()
            tu.append(a.elapsed_time(b))
        wu = shg.solve_batch_device(pu, None, None, stream=sptr)
        relu = np.abs(wu - p64) / np.abs(p64)
        mu = statistics.median(tu)
        unguarded = {"value": point_steps(pu) / (mu * 1e-3), "unit": "grid-pt·steps/s", "ms_per_step": mu,
                     "sh_power_rel_max": float(relu.max()), "sh_power_rel_median": float(np.median(relu)),
                     "instances_above_1e-5": int((relu > 1e-5).sum())}

    out = {
        "metric": "batched SSFM grid-pt·steps/s",
        "value": value,
        "unit": "grid-pt·steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms,
        "higher_is_better": True,
        "scaling": args.scaling,
        "vs_baseline": None,
        "dtype": "f32" if args.precision == 32 else "f64",
        "data": "synthetic (seeded parameter sweep; fields generated on device from the parameters)",
        "config": {
            "workload": "batched plain SSFM sweep, 256 instances, seed = rank" if args.scaling == "weak" else
                        f"batched plain SSFM sweep, 256 instances (seed 0) split over {world} ranks",
            "instances": len(ps), "grid_sides": [64, 128, 192, 256], "nz_range": [100, 400],
            "point_steps_per_gpu": pts, "precision": args.precision,
            "l2": "a 256 MB buffer is written between timed steps (L2 flushed); fields stay in shared memory",
            "schedule": tuned or "compiled defaults",
        },
        "e2e": {"value": e2e_value, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "ms_per_step": e2e_ms},
        # one persistent launch per (precision the instance runs in, grid side) group per step
        "gpu_launches": args.steps * len({(64 if (p.fp32_guard > 0 and shg.fp32_error_estimate(p) > p.fp32_guard)
                                           else p.precision, p.nx) for p in ps}),
        "roofline": {"bound": "fp32-issue" if args.precision == 32 else "fp64-issue", "achieved": achieved_tflops,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved_tflops / peak,
                     "traffic": SWEEP_256_DRAM_BYTES_PER_LAUNCH if (args.precision == 32 and not args.class_side) else None,
                     "traffic_note": "DRAM bytes per launch of the 256x256 FP32 class, ncu capture of this bench",
                     "peak_source": f"nominal {B200_SMS} SMs x {lanes} lanes x 2 flop x measured median SM clock {sm_mhz:.0f} MHz",
                     "kernel": f"ssfm_plain_kernel, {nmax}x{nmax} class ({len(dom)} FP32 instances), one launch, "
                               + next((f"{t['cluster']}-CTA clusters x {t['threads']} threads (tuned)"
                                       for t in tuned if t["n"] == nmax), "compiled default split"),
                     "launch_ms": dom_ms, "flops_per_launch": algorithmic_flops(dom),
                     "sweep": {"achieved": sweep_tflops, "frac": sweep_tflops / peak, "flops": fl,
                               "note": "all four classes, concurrent on forked streams"},
                     "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
                             "note": "32 B/pt-step algorithmic (FP32) against measured copy bandwidth; the fields do not touch HBM between steps"}},
        "clocks": clocks,
    }
    if err is not None:
        out["fp32_error_vs_fp64"] = err
    if unguarded is not None:
        out["fp32_unguarded"] = unguarded
    if args.precision == 32 and args.fp32_guard > 0:
        prom = [p for p in ps if shg.fp32_error_estimate(p) > args.fp32_guard]
        out["config"]["fp32_guard"] = {
            "guard": args.fp32_guard, "instances_on_fp64_march": len(prom),
            "point_steps_on_fp64_march_frac": point_steps(prom) / point_steps(ps),
            "note": "instances whose predicted FP32 SH field error (shg_fp32_error_estimate) exceeds the guard "
                    "run the FP64 march with FP32 outputs; the rest, and all transforms of the rest, run in FP32"}
    if world == 1 and not args.class_side and args.precision == 32 and not args.no_extras:
        # the rest of the metric: the plain per-instance FP64 path on the same sweep, and the
        # adjoint gradients of the 256 x 256 / nz = 400 configuration
        out["fp64_plain_per_instance"] = fp64_per_instance(ps, value)
        out["adjoint"] = adjoint_figures(32, args.adjoint_batch, 5, 3, args.checkpoint_every)
        try:
            out["thermal_batch_8x512x512x1000"] = thermal_batch_512_figures()
        except Exception as e:  # the sweep line stands without it
            out["thermal_batch_8x512x512x1000"] = {"error": str(e)[:300]}
        try:
            out["thermal_128x128x200"] = thermal_128_figures()
        except Exception as e:
            out["thermal_128x128x200"] = {"error": str(e)[:300]}
    if args.class_side:
        out["config"]["workload"] = f"{len(ps)} instances of {args.class_side}x{args.class_side}, nz = {args.class_nz}"
    if not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(ps, args.precision)
    return out


def thermal_batch_512_figures() -> dict:
    """The large thermal batch as stated: 8 thermal runs of 512x512 / nz = 1000 in FP32 (50 W,
    w0 = 50 µm, 20 mm, ovens evenly spaced 30-65 °C), each to max|ΔT| < 1e-6 K in every one of
    at most 5 outer iterations, with dJ/dT_oven through the temperature field, in one
    shg_thermal_batch call; each outer iteration's heat equation is solved to the Jacobi sweeps'
    fixed point directly (heat_solver = SHG_HEAT_DIRECT) and checked by one FP64 sweep.  Device
    time by CUDA events, after a two-instance warm-up."""
    import torch
    from cushg_b200 import shg

    ps = [p.replace(precision=32, heat_solver=P.SHG_HEAT_DIRECT) for p in P.config_thermal_512(8)]
    shg.reserve_device_memory((12 << 30) * len(ps) + (5 << 30))
    shg.thermal_batch([q.replace(max_outer=2, nz=20) for q in ps[:2]], grad=True)  # kernels, transforms
    torch.cuda.synchronize()
    stats, dt = shg.thermal_batch(ps, grad=True)
    torch.cuda.synchronize()
    return {"metric": "thermal batch time", "value": stats[0].device_ms, "unit": "ms",
            "workload": "8 x thermal 512x512x1000 FP32, max|dT| < 1e-6 K in each of <= 5 outer iterations, "
                        "dJ/dT_oven; heat equation solved to the Jacobi fixed point (direct, FP64)",
            "outer_iterations": [st.outer_iterations for st in stats],
            "max_check_sweep_dT_K": max(st.last_residual for st in stats),
            "heat_solve_ms_per_instance": statistics.median(st.jacobi_ms for st in stats),
            "optical_passes_ms": stats[0].optics_ms,
            "sh_power_w": [st.sh_power for st in stats],
            "dJ_dToven_w_per_k": [float(x) for x in dt]}


def thermal_128_figures() -> dict:
    """The thermal configuration as stated (128 x 128 x 200 FP64, 20 mm, 20 W, w0 = 40 µm, oven
    40 °C, max|ΔT| < 1e-6 K inside <= 5 outer iterations), one shg_solve_device call each way:
    with the reference's Jacobi sweeps (its bits and sweep counts) and with the direct heat
    solve (each outer iteration at the sweeps' fixed point).  Device times by CUDA events,
    after an untimed run of each."""
    import torch
    from cushg_b200 import shg

    p = P.config_thermal_128()
    pump = torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda")
    sig = torch.empty_like(pump)
    out = {"workload": "thermal 128x128x200 FP64, max|dT| < 1e-6 K, <= 5 outer iterations"}
    for name, q in (("jacobi", p), ("direct", p.replace(heat_solver=P.SHG_HEAT_DIRECT))):
        shg.solve_device(q, pump, sig)
        torch.cuda.synchronize()
        st = shg.solve_device(q, pump, sig)
        torch.cuda.synchronize()
        out[name] = {"device_ms": st.device_ms, "heat_ms": st.jacobi_ms, "optics_ms": st.optics_ms,
                     "jacobi_sweeps": st.jacobi_sweeps, "outer_iterations": st.outer_iterations,
                     "sh_power_w": st.sh_power}
    return out


def fp64_per_instance(ps, fp32_batch_value: float, count: int = 32) -> dict:
    """The plain FP64 path run per instance (one shg_solve_device call per instance, as the
    reference runs one process per point) over a stride sample of the sweep: pt-steps/s from
    the calls' device times, and the FP32 batch's rate over it."""
    import torch
    from cushg_b200 import shg

    sample = [p.replace(precision=64) for p in sample_stride(ps, count)]
    bufs = {}
    for p in sample:
        if p.nx not in bufs:
            bufs[p.nx] = (torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda"),
                          torch.empty((p.ny, p.nx), dtype=torch.complex128, device="cuda"))
    for p in sample[:4]:
        shg.solve_device(p, *bufs[p.nx])
    torch.cuda.synchronize()
    dev_ms = sum(shg.solve_device(p, *bufs[p.nx]).device_ms for p in sample)
    v = point_steps(sample) / (dev_ms * 1e-3)
    single = P.config_adjoint().replace(precision=64)
    b = (torch.empty((256, 256), dtype=torch.complex128, device="cuda"),
         torch.empty((256, 256), dtype=torch.complex128, device="cuda"))
    for _ in range(3):
        shg.solve_device(single, *b)
    t256 = statistics.median(shg.solve_device(single, *b).device_ms for _ in range(5))
    return {"value": v, "unit": "grid-pt·steps/s", "sample": f"{len(sample)} of the sweep's instances (stride), "
                                                               "one call each, summed device time",
            "fp32_batch_over_fp64_per_instance": fp32_batch_value / v,
            "n256_nz400_ms": t256, "n256_nz400_pt_steps_per_s": 256 * 256 * 399 / (t256 * 1e-3)}


def adjoint_figures(precision: int, batch: int, steps: int, warmup: int, checkpoint_every: int = 0,
                    nz: int = 0) -> dict:
    """Gradients of the SH power of the 256x256 / nz = 400 run (20 mm, 30 W, w0 = 35 µm, focus
    0.4 L, 30 °C) with respect to waist, focus, oven temperature and a 399-entry poling-phase
    vector drawn from N(0, 0.1 rad): a batch of `batch` such instances (poling seeds 0..B-1) in
    one shg_grad_batch call against the batched forward march of the same instances (both fill
    the GPU, so this is the cost ratio), and one instance's latency against its forward march.
    Medians of device times over `steps` runs after `warmup`."""
    import torch
    from cushg_b200 import shg

    p = P.config_adjoint().replace(precision=precision)
    if nz:
        p = p.replace(nz=nz)
    nst = p.nz - 1
    # the compiled schedules for both the gradients and the forward they are compared with
    # (a schedule tuned for the mixed sweep is not this batch's)
    shg.autotune_reset()
    kk = checkpoint_every
    cdt = torch.complex64 if p.precision == 32 else torch.complex128

    def polv(seed):
        return np.random.default_rng(seed).normal(0.0, 0.1, size=nst)

    # single instance: latency
    pol = polv(0)
    for _ in range(warmup):
        shg.grad(p, pol, checkpoint_every=kk)
    g_ms = []
    for _ in range(steps):
        g = shg.grad(p, pol, checkpoint_every=kk)
        g_ms.append(g["device_ms"])
    pump = torch.empty((p.ny, p.nx), dtype=cdt, device="cuda")
    sig = torch.empty_like(pump)
    for _ in range(warmup):
        shg.solve_device(p, pump, sig)
    f_ms = [shg.solve_device(p, pump, sig).device_ms for _ in range(steps)]
    gm, fm = statistics.median(g_ms), statistics.median(f_ms)

    # batch: throughput and cost ratio
    ps = [p] * batch
    pols = [polv(i) for i in range(batch)]
    for _ in range(max(1, warmup - 2)):
        shg.grad_batch(ps, pols, checkpoint_every=kk)
    gbr = [shg.grad_batch(ps, pols, checkpoint_every=kk)[0] for _ in range(steps)]
    gb = [r["device_ms"] for r in gbr]
    pumps = [torch.empty((p.ny, p.nx), dtype=cdt, device="cuda") for _ in range(batch)]
    sigs = [torch.empty_like(t) for t in pumps]
    stream = torch.cuda.current_stream()
    for _ in range(warmup):
        shg.solve_batch_device(ps, pumps, sigs, stream=stream.cuda_stream, want_power=False)
    torch.cuda.synchronize()
    fb = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        shg.solve_batch_device(ps, pumps, sigs, stream=stream.cuda_stream, want_power=False)
        b.record(stream)
        torch.cuda.synchronize()
        fb.append(a.elapsed_time(b))
    gbm, fbm = statistics.median(gb), statistics.median(fb)
    return {"value": batch * 1e3 / gbm, "unit": "gradients/s",
            "workload": f"{batch} x (256x256 nz={p.nz}, 3 scalars + {nst}-vector), checkpoints every "
                        f"{gbr[0]['checkpoint_every']} steps (single gradient: every {g['checkpoint_every']})",
            "precision": p.precision, "batch": batch, "batch_grad_ms": gbm, "batch_forward_ms": fbm,
            "grad_over_forward": gbm / fbm,
            "single": {"grad_ms": gm, "forward_ms": fm, "grad_over_forward": gm / fm},
            "sh_power_w": g["sh_power"], "d_waist": g["d_waist"], "d_focus": g["d_focus"], "d_temp": g["d_temp"]}


def cpu_baseline(ps, precision: int, count: int = 24) -> dict:
    """The CPU restatement (oracle/) on every host core over a stride sample of the sweep."""
    from oracle import oracle as O

    sample = sample_stride(ps, count)
    cores = os.cpu_count() or 1
    O.lib()
    t0 = time.perf_counter()
    O.batch_plain(sample, nthreads=cores)
    dt = time.perf_counter() - t0
    pts = point_steps(sample)
    return {"value": pts / dt, "unit": "grid-pt·steps/s", "cores": cores, "kind": "port",
            "sample": f"{len(sample)} of the 256 instances (every {max(1, len(ps) // count)}th), full nz, "
                      f"precision {precision}, {pts:.3g} pt-steps in {dt:.1f} s"}


# -------------------------------------------------------------------- reference (CPU) arm
def run_reference(args, rank: int, world: int) -> dict | None:
    if rank != 0:
        return None
    from oracle import oracle as O

    ps = P.config_sweep(256, seed=0, precision=32)
    sample = sample_stride(ps, 24)
    cores = os.cpu_count() or 1
    O.lib()
    for _ in range(args.warmup):
        O.batch_plain(sample[:cores], steps=[4] * min(cores, len(sample)), nthreads=cores)
    pts = point_steps(sample)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        O.batch_plain(sample, nthreads=cores)
        times.append(time.perf_counter() - t0)
    dt = sum(times) / len(times)
    v = pts / dt
    return {
        "impl": "reference", "metric": "batched SSFM grid-pt·steps/s", "value": v, "unit": "grid-pt·steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded parameter sweep)",
        "config": {"workload": "batched plain SSFM sweep, 256 instances, seed 0 (stride sample of 24 per step)",
                   "instances": len(sample), "precision": 32},
        "cpu_baseline": {"value": v, "unit": "grid-pt·steps/s", "cores": cores, "kind": "port",
                         "sample": f"{len(sample)} of 256 instances (every {len(ps) // 24}th), full nz, FP32 restatement "
                                   f"of the reference (the reference itself is CUDA-only)"},
        "e2e": {"value": v, "unit": "grid-pt·steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_thermal(args) -> dict:
    """Thermal workload (outside the default sweep line): one full thermal solve of the
    128x128 / nz = 200 FP64 configuration (20 mm, 20 W, w0 = 40 µm, oven 40 °C, Jacobi to
    max|ΔT| < 1e-6 K inside <= 5 outer iterations), timed with CUDA events."""
    import torch
    from cushg_b200 import shg

    p = P.config_thermal_128()
    if args.thermal_side:
        p = p.replace(nx=args.thermal_side, ny=args.thermal_side)
    if args.thermal_nz:
        p = p.replace(nz=args.thermal_nz)
    if args.thermal_max_sweeps:
        p = p.replace(max_sweeps=args.thermal_max_sweeps)
    direct = args.heat_solver == "direct"
    p = p.replace(jacobi_block=args.jacobi_block, precision=args.thermal_precision or 64,
                  heat_solver=P.SHG_HEAT_DIRECT if direct else P.SHG_HEAT_JACOBI,
                  march={"auto": P.SHG_MARCH_AUTO, "fused": P.SHG_MARCH_FUSED,
                         "multipass": P.SHG_MARCH_MULTIPASS}[args.march])
    cdt = torch.complex128 if p.precision == 64 else torch.complex64
    if direct:  # operator transforms (computed once per process) and kernels before timing
        wp = torch.empty((p.ny, p.nx), dtype=cdt, device="cuda")
        shg.solve_device(p.replace(max_outer=1), wp, torch.empty_like(wp))
    pump = torch.empty((p.ny, p.nx), dtype=cdt, device="cuda")
    sig = torch.empty_like(pump)
    with ClockSampler(0) as clk:
        t0 = time.perf_counter()
        try:
            st = shg.solve_device(p, pump, sig)
            status = "ok"
        except shg.ShgError as e:  # e.g. the sweep cap
            st, status = None, str(e)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    vox = p.nx * p.ny * p.nz
    out = {"metric": "thermal solve (Jacobi voxel-sweeps/s)",
           "workload": f"thermal {p.nx}x{p.ny}x{p.nz} FP{p.precision}", "status": status,
           "jacobi_block": p.jacobi_block or "auto (1)", "wall_s": wall, "clocks": clk.summary()}
    if st is not None and direct:
        out.update({"metric": "thermal solve time", "heat_solver": "direct", "value": st.device_ms, "unit": "ms",
                    "higher_is_better": False, "device_ms": st.device_ms, "heat_solve_ms": st.jacobi_ms,
                    "optics_ms": st.optics_ms, "outer_iterations": st.outer_iterations, "sh_power_w": st.sh_power,
                    "last_max_dT_K": st.last_residual,
                    "note": "each outer iteration's temperature is the Jacobi sweeps' fixed point; last_max_dT_K "
                            "is max |ΔT| of one FP64 sweep applied to the last one"})
        out.pop("jacobi_block")
    elif st is not None:
        out.update({"device_ms": st.device_ms, "jacobi_ms": st.jacobi_ms, "optics_ms": st.optics_ms,
                    "jacobi_sweeps": st.jacobi_sweeps, "outer_iterations": st.outer_iterations,
                    "sh_power_w": st.sh_power, "value": vox * st.jacobi_sweeps / (st.device_ms * 1e-3),
                    "unit": "voxel-sweeps/s",
                    "jacobi_gbs_algorithmic": 3 * (p.precision // 8) * vox * st.jacobi_sweeps / (st.device_ms * 1e-3) / 1e9})
    return out


def run_thermal_batch(args) -> dict:
    """Large thermal batch (outside the default sweep line): `--thermal-count` instances of
    512x512 / nz = 1000 in FP32 (50 W, w0 = 50 µm, 20 mm, ovens evenly spaced 30-65 °C), each a
    full thermal run through shg_solve_device with a fixed cost per optical-thermal update:
    `--thermal-fixed-sweeps` Jacobi sweeps (FP64 residual of the last one reported) in each of
    `--thermal-outer` outer iterations.  Jacobi to max|ΔT| < 1e-6 K at this size needs on the
    order of 1e6 sweeps per outer iteration, beyond a bench budget.  Each instance also gets
    dJ/dT_oven through its temperature field, unless --no-thermal-grad.  `--thermal-mode batch`
    (default): all instances in one shg_thermal_batch call (optical and tangent passes batched);
    `sequential`: one shg_solve_device / shg_thermal_grad call per instance."""
    import torch
    from cushg_b200 import shg

    # each 512 x 512 x 1000 FP32 instance uses about 11 GB of workspace: keep it in the
    # library's pool from one instance to the next (read when the pool is first created), and
    # grow the pool to it before the timed runs (set-up, as an application would at start)
    ps = P.config_thermal_512(args.thermal_count)
    if args.thermal_nz:  # a shorter crystal grid, e.g. for a launch list
        ps = [p.replace(nz=args.thermal_nz) for p in ps]
    direct = args.heat_solver == "direct"
    if direct:  # the stated rule: max|ΔT| < 1e-6 K every outer iteration, at most 5 of them
        ps = [p.replace(precision=32, heat_solver=P.SHG_HEAT_DIRECT) for p in ps]
        label = (f"{len(ps)} x thermal 512x512x{ps[0].nz} FP32, heat equation solved to the Jacobi fixed point "
                 f"(direct, FP64) every outer iteration, <= {ps[0].max_outer} outer iterations, "
                 f"max|ΔT| < {ps[0].jacobi_tol:g} K")
    else:
        ps = [p.replace(conv_rule=P.SHG_CONV_FIXED, max_sweeps=args.thermal_fixed_sweeps,
                        max_outer=args.thermal_outer, precision=32) for p in ps]
        label = (f"{len(ps)} x thermal 512x512x{ps[0].nz} FP32, {args.thermal_outer} outer x "
                 f"{args.thermal_fixed_sweeps} Jacobi sweeps each")
    if args.thermal_mode == "batch":
        # all instances in one shg_thermal_batch call: every instance's buffers and tangent at
        # once (about 11.5 GB each at 512 x 512 x 1000 FP32), in the pool before timing
        extra = (5 << 30) if direct else 0  # the direct solve's two FP64 volumes (4.2 GB)
        os.environ.setdefault("SHG_POOL_KEEP_MB", str(12 * 1024 * len(ps) + 4096 + (extra >> 20)))
        shg.reserve_device_memory((12 << 30) * len(ps) + extra)
        grad = not args.no_thermal_grad
        for _ in range(1):  # warm-up on two instances: kernel loading, pool growth, operator transforms
            shg.thermal_batch([q.replace(max_sweeps=2, max_outer=2, nz=20) for q in ps[:2]], grad=grad)
            if direct:
                shg.thermal_batch([ps[0].replace(max_outer=1, nz=20)], grad=False)
        torch.cuda.synchronize()
        with ClockSampler(0) as clk:
            t0 = time.perf_counter()
            stats, dt = shg.thermal_batch(ps, grad=grad)
            torch.cuda.synchronize()
            wall_ms = 1e3 * (time.perf_counter() - t0)
        runs = []
        for i, (p, st) in enumerate(zip(ps, stats)):
            r = {"oven_c": round(p.temp, 2), "sh_power_w": st.sh_power, "sweeps": st.jacobi_sweeps,
                 "outer_iterations": st.outer_iterations, "jacobi_ms": st.jacobi_ms, "optics_ms": st.optics_ms,
                 "last_max_dT_K": st.last_residual}
            if dt is not None:
                r["dJ_dToven_w_per_k"] = float(dt[i])
            runs.append(r)
        return {"metric": "thermal batch time", "value": stats[0].device_ms, "unit": "ms", "higher_is_better": False,
                "timing": "device time of one shg_thermal_batch call (CUDA events)", "wall_ms": wall_ms,
                "mode": "batch", "with_gradient": grad, "heat_solver": args.heat_solver, "workload": label,
                "max_last_dT_K": max(st.last_residual for st in stats), "instances": runs, "clocks": clk.summary()}
    os.environ.setdefault("SHG_POOL_KEEP_MB", "16384")
    shg.reserve_device_memory(12 << 30)

    def one(p):
        if args.no_thermal_grad:
            pump = torch.empty((p.ny, p.nx), dtype=torch.complex64, device="cuda")
            sig = torch.empty_like(pump)
            st = shg.solve_device(p, pump, sig)
            torch.cuda.synchronize()
            return ({"oven_c": round(p.temp, 2), "sh_power_w": st.sh_power, "device_ms": st.device_ms,
                     "jacobi_ms": st.jacobi_ms, "optics_ms": st.optics_ms,
                     "sweeps": st.jacobi_sweeps, "last_max_dT_K": st.last_residual}, st.jacobi_sweeps,
                    st.outer_iterations)
        g = shg.thermal_grad(p)
        # jacobi_ms: the forward run's heat solve; optics_ms: its per-voxel optics and optical
        # marches; the rest of device_ms is the tangent (its own sweeps included)
        return ({"oven_c": round(p.temp, 2), "sh_power_w": g["sh_power"], "dJ_dToven_w_per_k": g["d_temp"],
                 "device_ms": g["device_ms"], "jacobi_ms": g["jacobi_ms"], "optics_ms": g["optics_ms"],
                 "sweeps": g["jacobi_sweeps"]}, g["jacobi_sweeps"], g["outer_iterations"])

    # --thermal-concurrency K: K instances at a time from K host threads (the library is
    # thread-safe and each call runs on its own stream), so one instance's optical marches,
    # which leave most SMs idle at 512 x 512, overlap another's Jacobi sweeps
    import concurrent.futures as cf
    with ClockSampler(0) as clk:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.thermal_concurrency > 1:
            with cf.ThreadPoolExecutor(max_workers=args.thermal_concurrency) as ex:
                out = list(ex.map(one, ps))
        else:
            out = [one(p) for p in ps]
        torch.cuda.synchronize()
        wall_ms = 1e3 * (time.perf_counter() - t0)
    runs = [r for r, _, _ in out]
    jac_vox = sum(float(p.nx * p.ny * p.nz) * sw for p, (_, sw, _) in zip(ps, out))
    opt_pts = sum(float(p.nx * p.ny * p.nz) * o for p, (_, _, o) in zip(ps, out))
    total_ms = sum(r["device_ms"] for r in runs)
    return {"metric": "thermal batch time", "value": wall_ms if args.thermal_concurrency > 1 else total_ms,
            "unit": "ms", "higher_is_better": False,
            "timing": ("wall clock of the whole batch, instances overlapping" if args.thermal_concurrency > 1
                       else "sum of the instances' device times, one at a time"),
            "concurrency": args.thermal_concurrency, "sum_device_ms": total_ms, "wall_ms": wall_ms,
            "workload": label, "heat_solver": args.heat_solver,
            "instances": runs, "voxel_sweeps": jac_vox, "optical_point_steps": opt_pts,
            "clocks": clk.summary()}


def run_heat_direct(args) -> dict:
    """Direct heat-solve workload (outside the default sweep line): shg_heat_steady_device on
    the large thermal batch's grid (512 x 512 x 1000, FP32 storage, FP64 solve, top-open
    boundary; --thermal-side / --thermal-nz / --thermal-precision change it) with a random heat
    source, timed with CUDA events on the launching stream.  Its four transform GEMMs carry
    2 (mx + my) 2 mx my nz FP64 flops, 2 nz mx my (mx + 2 my) with the folded x transform; for scale, cuBLAS's FP64 matmul (torch.matmul) is timed
    on the x-transform's shape, the same flops in one call."""
    import torch
    from cushg_b200 import shg

    p = P.config_thermal_512(1)[0]
    if args.thermal_side:
        p = p.replace(nx=args.thermal_side, ny=args.thermal_side)
    if args.thermal_nz:
        p = p.replace(nz=args.thermal_nz)
    p = p.replace(precision=args.thermal_precision or 32)
    n, nz = p.nx, p.nz
    # the solve's two FP64 volumes stay in the library's pool from call to call
    work = 2 * 8 * n * n * nz + (64 << 20)
    os.environ.setdefault("SHG_POOL_KEEP_MB", str((work >> 20) + 1024))
    shg.reserve_device_memory(work)
    tdt = torch.float64 if p.precision == 64 else torch.float32
    g = torch.Generator(device="cuda").manual_seed(0)
    Q = (torch.rand((nz, n, n), dtype=torch.float64, device="cuda", generator=g) * (60.0 * p.kappa / p.lx ** 2)).to(tdt)
    T0 = torch.full((nz, n, n), p.temp, dtype=tdt, device="cuda")
    T0[:, 0, :] = p.t_peltier  # top-open: the y = 0 face at the oven temperature
    T = T0.clone()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    for _ in range(max(1, args.warmup)):
        T.copy_(T0)
        resid = shg.heat_steady_device(p, T, Q, stream=sptr)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for a, b in evs:
            a.record(stream)
            shg.heat_steady_device(p, T, Q, stream=sptr)
            b.record(stream)
        torch.cuda.synchronize()
    ms = statistics.median(x.elapsed_time(y) for x, y in evs)
    mx, my = n, n - 1
    unfolded = 2.0 * (mx + my) * 2.0 * mx * my * nz
    # top-open x is Robin at both ends: with mx a multiple of 4 the x transforms run folded
    # (even and odd modes from half-size products), half the x flops
    flops = 2.0 * nz * mx * my * (mx + 2.0 * my) if mx % 4 == 0 else unfolded
    # cuBLAS FP64 on the x-transform's shape (nz*my x mx) @ (mx x mx), scaled to all four GEMMs
    A = torch.rand((nz * my, mx), dtype=torch.float64, device="cuda", generator=g)
    B = torch.rand((mx, mx), dtype=torch.float64, device="cuda", generator=g)
    for _ in range(3):
        C = A @ B
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(5):
        C = A @ B
    e1.record(stream)
    torch.cuda.synchronize()
    cublas_tflops = 5 * 2.0 * A.shape[0] * mx * mx / (e0.elapsed_time(e1) * 1e-3) / 1e12
    del A, B, C
    return {"metric": "direct heat solve time", "value": ms, "unit": "ms", "higher_is_better": False,
            "workload": f"shg_heat_steady_device {n}x{n}x{nz} FP{p.precision} storage, FP64 solve",
            "residual_max_dT_K": resid, "gemm_tflop_per_solve": flops / 1e12,
            "gemm_tflop_per_solve_unfolded": unfolded / 1e12,
            "gemm_tflops_if_all_time": flops / (ms * 1e-3) / 1e12,
            "cublas_fp64_matmul_tflops_same_shape": cublas_tflops,
            "note": "gemm_tflops_if_all_time divides the transform flops by the whole solve's time "
                    "(right-hand side, tridiagonal pass and finish included)",
            "clocks": clk.summary()}


def run_jacobi(args) -> dict:
    """Heat-solve workload (outside the default sweep line): `--jacobi-sweeps` Jacobi sweeps
    of the heat equation per step through shg_heat_sweeps_device on the thermal grid (default
    128 x 128 x 200, FP64, top-open boundary), from a uniform 40 °C start with a random heat
    source; timed with CUDA events on the launching stream."""
    import torch
    from cushg_b200 import shg

    p = P.config_thermal_128()
    if args.thermal_side:
        p = p.replace(nx=args.thermal_side, ny=args.thermal_side)
    if args.thermal_nz:
        p = p.replace(nz=args.thermal_nz)
    p = p.replace(jacobi_block=args.jacobi_block, precision=args.thermal_precision or 64)
    tdt = torch.float64 if p.precision == 64 else torch.float32
    vox = p.nx * p.ny * p.nz
    T = torch.full((p.nz, p.ny, p.nx), 40.0, dtype=tdt, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(0)
    Q = torch.rand((p.nz, p.ny, p.nx), dtype=tdt, device="cuda", generator=g) * 1e-6
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    k = args.jacobi_sweeps
    for _ in range(args.warmup):
        shg.heat_sweeps_device(p, T, Q, k, stream=sptr)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for a, b in evs:
            a.record(stream)
            shg.heat_sweeps_device(p, T, Q, k, stream=sptr)
            b.record(stream)
        torch.cuda.synchronize()
    ms = statistics.median(x.elapsed_time(y) for x, y in evs)
    per_sweep_s = ms * 1e-3 / k
    bpv = 3 * (p.precision // 8)
    hbm_peak = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else 6650.0
    gbs = bpv * vox / per_sweep_s / 1e9
    return {"metric": "Jacobi voxel-sweeps/s", "value": vox / per_sweep_s, "unit": "voxel-sweeps/s",
            "workload": f"heat sweeps {p.nx}x{p.ny}x{p.nz} FP{p.precision}, {k} sweeps per call",
            "jacobi_block": args.jacobi_block, "ms_per_call": ms, "us_per_sweep": per_sweep_s * 1e6,
            "working_set_mb": 3 * vox * (p.precision // 8) / 1e6,
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": hbm_peak, "unit": "GB/s", "frac": gbs / hbm_peak,
                         "note": f"{bpv} B per voxel-sweep algorithmic (read T, read Q, write T); above 1.0 means "
                                 f"the sweep runs from L2 or fuses sweeps"},
            "clocks": clk.summary()}


def run_adjoint(args) -> dict:
    """Adjoint workload (outside the default sweep line; the default line carries the same
    figures under "adjoint"): see adjoint_figures.  value: gradients/s of a batch of
    `--adjoint-batch` instances in one shg_grad_batch launch."""
    r = adjoint_figures(args.precision, args.adjoint_batch, args.steps, args.warmup, args.checkpoint_every,
                        args.adjoint_nz)
    return {"metric": "adjoint grads/s", **r}


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fp32-guard", type=float, default=1e-5,
                    help="FP32 sweep: instances whose predicted FP32 SH field error exceeds this run the FP64 "
                         "march (0: all FP32)")
    ap.add_argument("--no-extras", action="store_true",
                    help="sweep line without the FP64 per-instance and adjoint figures (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="use the compiled default launch schedules (default: shg_autotune_batch on the workload)")
    ap.add_argument("--scaling", default="weak", choices=["weak", "strong"],
                    help="weak: every rank runs its own 256-instance sweep; strong: one sweep split over the ranks")
    ap.add_argument("--class-side", type=int, default=0, help="profile case: one grid-size class only")
    ap.add_argument("--class-count", type=int, default=18)
    ap.add_argument("--class-nz", type=int, default=24)
    ap.add_argument("--class-schedule", default="",
                    help="with --class-side: the compiled split to use, as CLUSTER,THREADS (shg_set_schedule)")
    ap.add_argument("--workload", default="sweep",
                    choices=["sweep", "thermal", "adjoint", "jacobi", "thermal-batch", "heat-direct"])
    ap.add_argument("--thermal-count", type=int, default=8)
    ap.add_argument("--thermal-fixed-sweeps", type=int, default=200)
    ap.add_argument("--thermal-outer", type=int, default=2)
    ap.add_argument("--no-thermal-grad", action="store_true", help="thermal-batch: the runs without dJ/dT_oven")
    ap.add_argument("--thermal-concurrency", type=int, default=1,
                    help="thermal-batch, sequential mode: instances run at a time from host threads")
    ap.add_argument("--thermal-mode", default="batch", choices=["batch", "sequential"],
                    help="thermal-batch: one shg_thermal_batch call, or one run per instance")
    ap.add_argument("--jacobi-sweeps", type=int, default=400)
    ap.add_argument("--thermal-side", type=int, default=0)
    ap.add_argument("--thermal-nz", type=int, default=0)
    ap.add_argument("--march", default="auto", choices=["auto", "fused", "multipass"],
                    help="optical march of the thermal workload")
    ap.add_argument("--checkpoint-every", type=int, default=0,
                    help="adjoint checkpoint interval (0: the library's choice)")
    ap.add_argument("--adjoint-nz", type=int, default=0, help="adjoint workload with this nz (profiling case)")
    ap.add_argument("--adjoint-batch", type=int, default=18, help="instances of the batched gradient")
    ap.add_argument("--thermal-max-sweeps", type=int, default=0)
    ap.add_argument("--thermal-precision", type=int, default=None, choices=[32, 64],
                    help="thermal, jacobi: default 64; heat-direct: default 32")
    ap.add_argument("--jacobi-block", type=int, default=0, help="sweeps per launch (0 = automatic)")
    ap.add_argument("--heat-solver", default="jacobi", choices=["jacobi", "direct"],
                    help="thermal workloads: Jacobi sweeps as the reference runs them, or their fixed point "
                         "solved directly each outer iteration")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.workload == "thermal":
        out = run_thermal(args) if rank == 0 else None
    elif args.workload == "adjoint":
        out = run_adjoint(args) if rank == 0 else None
    elif args.workload == "jacobi":
        out = run_jacobi(args) if rank == 0 else None
    elif args.workload == "thermal-batch":
        out = run_thermal_batch(args) if rank == 0 else None
    elif args.workload == "heat-direct":
        out = run_heat_direct(args) if rank == 0 else None
    elif args.impl == "reference":
        out = run_reference(args, rank, world)
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
