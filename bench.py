"""Benchmark of the AutoGrid4 map hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference] [--workload NAME]

Metric: grid-point x map-type evaluations per second (P * M / time) for the
plain large map set: a seeded synthetic 10,000-atom receptor in a 45 A sphere,
npts 126^3 (127^3 = 2,048,383 points), 14 ligand types + e + d = 16 maps,
spacing 0.375 A, distance-dependent dielectric.  One step = one full map set.

  value    device-resident: ag_plan_run over inputs already in HBM; L2 is
           flushed (256 MiB write) before every timed step; CUDA events.
  e2e      the public C ABI call ag_maps_compute with host inputs and a pinned
           host output: host preparation, H2D, kernels and D2H every step.
  roofline the dominant kernel (far-field e map, k_emap_far): algorithmic pair
           terms per second (1 rsqrt each) against the measured MUFU rsqrt rate
           of this GPU.
  cpu_baseline  the reference's own OpenMP build (oracle/_ref/autogrid4,
           compiled from the reference sources) on a bounded sample of the same
           workload: same receptor and 16 maps, fewer z-planes.

Multi-GPU (torchrun, one process per GPU): the one map set is split by
z-slab (autogrid_b200.shard.zslab_ranges; ag_plan_run_zslab for `value`,
ag_maps_compute_zslab for `e2e`), strong scaling: total work fixed, time =
max over ranks, no collective on the data path (the timing reduction is the
only one).  The batched ensemble splits by instance (shard.partition_instances).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import shutil
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "ad4_10000_127cube_16maps"
METRIC = "grid-pt*type evals/s (plain 127^3 x 16-map AD4 set, 10k-atom receptor)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-ensemble comparison")
    ap.add_argument("--batch-instances", type=int, default=256)
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable-mode measurement")
    ap.add_argument("--no-vina", action="store_true", help="skip the batched Vina conformer measurement")
    ap.add_argument("--no-text", action="store_true", help="skip the device map-text measurement")
    ap.add_argument("--vina-conformers", type=int, default=32,
                    help="conformers of the batched Vina measurement (fewer for a profiling case)")
    return ap.parse_args()


def max_over_ranks(values, world: int, device: str) -> list:
    """Each value's maximum over the ranks (the job's time is its slowest
    rank's); every rank gets the result.  One all-reduce, the only collective
    of the timed run; `device` is where the process group's backend reduces
    ("cuda" for NCCL, "cpu" for gloo)."""
    if world <= 1:
        return [float(v) for v in values]
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def dist_info():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        self.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits", "-lms", "100"],
                                     stdout=self.out, stderr=subprocess.DEVNULL)

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.flush()
        rows = [r.split(",") for r in Path(self.out.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.out.name)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx.append(float(r[2]))
            except (ValueError, IndexError):
                continue
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].strip().lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def make_problem(workload: str, seed: int, workdir: Path):
    from autogrid_b200 import Job, synth
    rec, spec = synth.workload(workload, seed=seed)
    gpf = synth.write_case(workdir, "bench", rec, spec)
    cwd = os.getcwd()
    os.chdir(workdir)
    try:
        job = Job(gpf.name, "bench.glg")
        prob = job.problem()
    finally:
        os.chdir(cwd)
    return rec, spec, job, prob


def reference_sample(rec, spec, workdir: Path, threads: int, nxy: int = 48):
    """Run the reference OpenMP binary on a centred sub-box of the workload
    (nxy x nxy x 4*threads npts; the reference hands out z-planes in blocks of
    4, schedule(static,4) at main.cpp:2805, so 4 planes per thread keeps every
    thread busy).  Returns (evals/s, seconds, points, maps, description)."""
    from autogrid_b200 import synth
    from oracle.oracle import REF_BIN
    if not REF_BIN.exists():
        return None
    nz = max(2, 4 * threads)
    sub = synth.GridSpec(npts=(nxy, nxy, nz), spacing=spec.spacing, ligand_types=list(spec.ligand_types))
    d = workdir / "ref"
    synth.write_case(d, "ref", rec, sub)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    t0 = time.perf_counter()
    r = subprocess.run([str(REF_BIN), "-p", "ref.gpf", "-l", "ref.glg"], cwd=d, env=env,
                       capture_output=True, text=True)
    dt = time.perf_counter() - t0
    if r.returncode != 0 or "Successful Completion" not in (d / "ref.glg").read_text():
        return None
    P = (sub.npts[0] + 1) * (sub.npts[1] + 1) * (nz + 1)
    M = len(spec.ligand_types) + 2
    glg = glg_times((d / "ref.glg").read_text())
    desc = (f"reference autogrid4 (OpenMP, {threads} threads, {cpu_model()}) on the same receptor and {M} maps, "
            f"npts {sub.npts[0]}x{sub.npts[1]}x{nz} ({P} points); whole-process wall time {dt:.2f} s, "
            f"GLG Real= total {glg['real_total_s']} s, sum of per-plane Real= {glg['plane_sum_s']} s "
            f"({glg['planes']} planes)")
    return P * M / dt, dt, P, M, desc


def glg_times(text: str) -> dict:
    """The reference log's timings: the per-plane 'Real= x.xx,' lines of its
    grid loop (timesys, main.cpp:3455) and the job's closing 'Real= [h] [m] s'
    (timesyshms, main.cpp:3568)."""
    planes, total = [], None
    for m in re.finditer(r"Real=\s*((?:(\d+)h\s*)?(?:(\d+)m\s*)?([0-9.]+)(s?)),", text):
        h, mi, sec, unit = m.group(2), m.group(3), float(m.group(4)), m.group(5)
        if unit == "s":
            total = (int(h or 0) * 3600 + int(mi or 0) * 60) + sec
        else:
            planes.append(sec)
    return {"real_total_s": total, "plane_sum_s": round(sum(planes), 3), "planes": len(planes)}


def cpu_model() -> str:
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "cpu model unknown"


def main():
    args = parse()
    rank, world, local = dist_info()
    if args.impl == "reference":
        return run_reference(args, rank, world)
    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    from autogrid_b200 import Context, load_library
    from autogrid_b200._abi import ag_stats  # noqa: F401

    work = Path(tempfile.mkdtemp(prefix=f"agb_bench_r{rank}_"))
    rec, spec, job, prob = make_problem(args.workload, seed=0, workdir=work)  # one map set, split over ranks
    P, M = prob.points, prob.n_maps
    from autogrid_b200.shard import zslab_ranges
    z0, z1 = zslab_ranges(prob.n1[2], world)[rank]
    slab_planes = z1 - z0
    ctx = Context(local)
    plan = ctx.plan(prob)

    def run_step():
        if world == 1:
            plan.run(sptr)
        elif slab_planes > 0:
            plan.run_zslab(z0, z1, sptr)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    # a dedicated stream: the library launches on it, and the events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    sptr = stream.cuda_stream
    assert sptr, "need a non-default CUDA stream"

    for _ in range(args.warmup):
        run_step()
    torch.cuda.synchronize()

    # ---------------- device-resident timed region ----------------
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    for k in range(args.steps):
        flush.zero_()
        starts[k].record(stream)
        run_step()
        ends[k].record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = float(np.mean(step_ms))
    plan.download()
    st = ctx.stats()
    launches_per_step = st.gpu_launches

    # dominant kernel alone: far-field e map (events around its launch), from a
    # plan that runs the same kernels in sequence on one stream -- in the timed
    # plan it overlaps the near-field kernel, so its own events span both
    lib = load_library()
    plan_serial = ctx.plan(prob, serial=True)
    ker = serial_kernel_ms(ctx, plan_serial, stream, args.steps)
    ker_ms = ker["far_ms"]
    plan_serial.close()

    # ---------------- end to end through the C ABI ----------------
    out_shape = prob.map_shape if world == 1 else (prob.n_out, slab_planes, prob.n1[1], prob.n1[0])
    out = torch.empty(out_shape, dtype=torch.float32, pin_memory=True).numpy()

    def e2e_step():
        if world == 1:
            ctx.compute(prob, "fp32", out=out)
        elif slab_planes > 0:
            ctx.compute_zslab(prob, z0, z1, out=out)

    e2e_step()  # warm the context's buffers
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e2e_t = []
    for k in range(args.steps):
        t0 = time.perf_counter()
        e2e_step()
        e2e_t.append(time.perf_counter() - t0)
    e2e_s = float(np.mean(e2e_t))

    ms, e2e_s = max_over_ranks([ms, e2e_s], world, "cuda")
    batch_sh = None
    if world > 1 and not args.no_batch:
        batch_sh = batched_sharded(ctx, args.batch_instances, work, stream, rank, world)

    if rank == 0:
        evals = P * M  # the whole map set, whatever the number of ranks
        rate_r, rate_f, clk_nominal = peak_rates(lib, local)
        pairs = prob.points * prob.n_atoms  # far-field pair terms (near pairs excluded are < 1%)
        achieved = pairs / (ker_ms * 1e-3) if ker_ms else None
        far_alone = ker_ms - ker["fixup_ms"]
        roof = {
            "bound": "sfu", "kernel": "k_emap_far + k_far_fixup (far-field e map with its bin guard)",
            "achieved": achieved / 1e9 if achieved else None, "peak": rate_r / 1e9 if rate_r else None,
            "unit": "Grsqrt/s", "frac": (achieved / rate_r) if (achieved and rate_r) else None,
            "traffic": profile_traffic("k_emap_far"),
            "peak_source": "measured on this GPU: rsqrt.approx.f32 microbenchmark (ag_diag_peak_rates)",
            "units_per_launch": f"{pairs} (point, atom) pair terms, 1 rsqrt each",
            "kernel_ms": ker_ms, "far_kernel_ms": far_alone, "fixup_ms": ker["fixup_ms"],
            "frac_far_kernel_alone": (pairs / (far_alone * 1e-3) / rate_r) if (rate_r and far_alone > 0) else None,
            "fp32_peak_tflops_measured": rate_f / 1e12 if rate_f else None,
        }
        # the near-field kernels: algorithmic FP32 flops of the in-range pairs
        # (12 per pair, 8 per ligand-map term, 2 for the d map, 13 for the e
        # term; directional H-bond terms not counted) against the measured
        # FP32 peak; they are latency-bound on their table-row loads
        n_lig = int(prob.scalars["n_atom_maps"])
        flops_pair = 12 + 8 * n_lig + 2 + 13
        near_flops = ker["near_pairs"] * flops_pair
        roof_near = {
            "bound": "fp32", "kernel": "k_near", "kernel_ms": ker["near_ms"],
            "achieved": near_flops / (ker["near_ms"] * 1e-3) / 1e12 if ker["near_ms"] else None,
            "peak": rate_f / 1e12 if rate_f else None, "unit": "TFLOP/s",
            "frac": (near_flops / (ker["near_ms"] * 1e-3) / rate_f) if (rate_f and ker["near_ms"]) else None,
            "traffic": profile_traffic("k_near"),
            "units_per_launch": f"{ker['near_pairs']} in-range (point, atom) pairs x {flops_pair} flops",
        }
        line = {
            "metric": METRIC, "value": evals / (ms * 1e-3), "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32 (FP64 fallback near table-bin edges)",
            "data": "synthetic (seeded receptor, shapes of the plain large map set)",
            "config": {"workload": args.workload, "atoms": prob.n_atoms, "points": P, "maps": M,
                       "npts": list(spec.npts), "spacing": spec.spacing,
                       "parallelism": "single GPU" if world == 1 else f"z-slab x{world}",
                       "l2": "flushed (256 MiB write) before every timed step"},
            "e2e": {"value": evals / e2e_s, "unit": "evals/s", "ms_per_step": e2e_s * 1e3,
                    "h2d_bytes_per_step": prob.bytes_h2d() * world, "d2h_bytes_per_step": P * M * 4},
            "gpu_launches": launches_per_step * args.steps,
            "roofline": roof,
            "roofline_near": roof_near,
            "clocks": clk,
            "diagnostics": {"near_pairs_per_step": st.near_pairs, "fp64_fallbacks_per_step": st.fp64_fallbacks,
                            "far_pairs_per_step": st.far_pairs,
                            # far-field bin guard: pairs resolved in FP64, of which the plain FP32
                            # bin was wrong, and FP64 ties decided by the reference expression
                            "far_edge_pairs_per_step": st.far_edge_pairs,
                            "far_fp32_bin_errors_per_step": st.far_fp32_bin_errors,
                            "far_fp64_ties_per_step": st.far_fp64_ties},
        }
        if batch_sh is not None:
            line["batched_sharded"] = batch_sh
        if not args.no_text and world == 1:
            line["map_text"] = map_text(ctx, plan, prob, rec, spec, work, args.steps)
        if not args.no_batch and world == 1:
            line["batched"] = batched_ensemble(ctx, args.batch_instances, work, stream)
        if not args.no_diff and world == 1:
            line["differentiable"] = differentiable_maps(ctx, work, stream)
        if not args.no_vina and world == 1:
            line["vina_conformers"] = vina_conformers(ctx, work, stream, K=args.vina_conformers)
        if world == 1:
            line["cli_e2e"] = cli_e2e(work, P * M)
        if not args.no_cpu_baseline and world == 1:
            threads = min(32, os.cpu_count() or 1)
            res = reference_sample(rec, spec, work, threads)
            if res:
                rate, dt, Ps, Ms, desc = res
                line["cpu_baseline"] = {"value": rate, "unit": "evals/s", "cores": threads,
                                        "kind": "reference", "sample": desc, "seconds": dt}
        print(json.dumps(line))
    plan.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    shutil.rmtree(work, ignore_errors=True)


def map_text(ctx, plan, prob, rec, spec, work: Path, steps: int):
    """The map-file text (main.cpp:3481-3519) of the same map set, formatted on
    the device from the plan's maps (ag_maps_format: measure, scan and write
    kernels, then one copy of the text to pinned host memory), and the whole
    one-shot call from host inputs to host text (ag_maps_compute_text).  The
    host writer (the reference's fprintf loop restated with snprintf, one
    thread) formats the same maps once for comparison."""
    from autogrid_b200 import Job, synth
    plan.run()
    for _ in range(2):
        mt = plan.format()
    fmt_s, kern_ms = [], []
    import torch
    for _ in range(steps):
        plan.run()
        torch.cuda.synchronize()  # the maps are done before the clock starts
        t0 = time.perf_counter()
        mt = plan.format()
        fmt_s.append(time.perf_counter() - t0)
        kern_ms.append(ctx.stats().text_ms)
    nbytes = mt.total
    one = []
    ctx.compute_text(prob)
    for _ in range(steps):
        t0 = time.perf_counter()
        ctx.compute_text(prob)
        one.append(time.perf_counter() - t0)
    maps = plan.download()
    d = work / "text_host"
    d.mkdir(exist_ok=True)
    g = synth.write_case(d, "bench", rec, spec)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        j = Job(g.name, None)
    finally:
        os.chdir(cwd)
    t0 = time.perf_counter()
    j.write_maps(maps)
    host_s = time.perf_counter() - t0
    j.close()
    shutil.rmtree(d, ignore_errors=True)
    values = prob.points * prob.n_out
    kms = float(np.median(kern_ms))
    alg = values * 4 + nbytes  # maps read once, text written once
    return {
        "text_bytes": nbytes, "values": values,
        "format_ms": float(np.median(fmt_s)) * 1e3,
        "format_kernels_ms": kms,
        "d2h_gbs": nbytes / (float(np.median(fmt_s)) - kms * 1e-3) / 1e9,
        "kernels_algorithmic_gbs": alg / (kms * 1e-3) / 1e9,
        "compute_text_ms": float(np.median(one)) * 1e3,
        "host_writer_s": host_s,
        "host_writer_note": "snprintf restatement of main.cpp:3481-3519, 1 thread, same maps",
        "speedup_vs_host_writer": host_s / (float(np.median(fmt_s))),
    }


def batched_ensemble(ctx, n, work: Path, stream):
    """The batched form: n uneven instances (atoms log-uniform 1,000-12,000,
    per-axis npts uniform 20-100, spacing 0.375 A, 8 maps) in one persistent,
    graph-captured launch per kernel kind, against the plain per-box path
    (one device-resident plan per instance, run one after another)."""
    import torch
    from autogrid_b200 import Batch, Job, load_library, synth
    d = work / "ensemble"
    gpfs = synth.write_ensemble(d, n, seed=2024)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        probs = [Job(os.path.basename(g), None).problem() for g in gpfs]
    finally:
        os.chdir(cwd)
    evals = sum(p.points * p.n_maps for p in probs)
    pairs = sum(p.points * p.n_atoms for p in probs)
    t0 = time.perf_counter()
    b = Batch(ctx, probs)
    create_s = time.perf_counter() - t0
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn, reps):
        out = []
        for _ in range(reps):
            flush.zero_()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            fn()
            e_.record(stream)
            torch.cuda.synchronize()
            out.append(s_.elapsed_time(e_))
        return float(np.mean(out))

    b.run(stream.cuda_stream)
    torch.cuda.synchronize()
    batch_ms = timed(lambda: b.run(stream.cuda_stream), 5)
    plans = [ctx.plan(p) for p in probs]
    near_pairs = 0
    for pl in plans:
        pl.run(stream.cuda_stream)
        near_pairs += ctx.stats().near_pairs
    torch.cuda.synchronize()
    plain_ms = timed(lambda: [pl.run(stream.cuda_stream) for pl in plans], 3)
    # same maps from both paths
    worst = 0.0
    for i in range(0, n, max(1, n // 16)):
        a = b.download(i)
        c = plans[i].download()
        worst = max(worst, float(np.max(np.abs(a - c) / np.maximum(1e-3, 1e-4 * np.abs(c)))))
    for pl in plans:
        pl.close()
    tune = b.tuning()
    b.close()
    # end to end through the public calls, host inputs and host maps: the
    # drop-in ag_maps_compute per box vs one ag_maps_compute_batch call, both
    # into the same pinned host arrays (touched once before timing, so no
    # first-touch page faults are timed)
    from autogrid_b200.api import compute_batch
    outs = [torch.empty(p.map_shape, dtype=torch.float32, pin_memory=True).numpy() for p in probs]
    for o in outs:
        o.fill(0.0)
    e2e_plain, e2e_batch = [], []
    for _ in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for p, o in zip(probs, outs):
            ctx.compute(p, "fp32", out=o)
        e2e_plain.append(time.perf_counter() - t0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        compute_batch(ctx, probs, outs)
        e2e_batch.append(time.perf_counter() - t0)
    e2e_plain_s, e2e_batch_s = min(e2e_plain), min(e2e_batch)
    cached = ctx.cached_bytes()  # device blocks the context keeps for later batch calls
    # roofline of the persistent kernels, timed alone by the autotuner: far
    # field (with its fix-up) against the measured rsqrt rate, near field as
    # algorithmic FP32 flops (as for the single map set) against the FP32 peak
    rate_r, rate_f, _ = peak_rates(load_library(), torch.cuda.current_device())
    lig = sum(int(p.scalars["n_atom_maps"]) for p in probs) / len(probs)
    near_flops = near_pairs * (12 + 8 * lig + 2 + 13)
    roof = {"far": {"kernel": "k_emap_far_batch + k_far_fixup_batch", "bound": "sfu", "kernel_ms": tune["far_ms"],
                    "achieved": pairs / (tune["far_ms"] * 1e-3) / 1e9, "unit": "Grsqrt/s",
                    "peak": rate_r / 1e9 if rate_r else None,
                    "frac": pairs / (tune["far_ms"] * 1e-3) / rate_r if rate_r else None},
            "near": {"kernel": "k_near_batch", "bound": "fp32", "kernel_ms": tune["near_ms"],
                     "achieved": near_flops / (tune["near_ms"] * 1e-3) / 1e12, "unit": "TFLOP/s",
                     "peak": rate_f / 1e12 if rate_f else None,
                     "frac": near_flops / (tune["near_ms"] * 1e-3) / rate_f if rate_f else None,
                     "near_pairs": int(near_pairs)}}
    return {"instances": n, "points": int(sum(p.points for p in probs)), "pair_terms": int(pairs),
            "roofline": roof,
            "e2e_plain_per_box_s": e2e_plain_s, "e2e_batch_s": e2e_batch_s,
            "e2e_speedup_vs_plain_per_box": e2e_plain_s / e2e_batch_s,
            "evals_per_s": evals / (batch_ms * 1e-3), "ms_per_ensemble": batch_ms,
            "plain_per_box_ms": plain_ms, "plain_per_box_evals_per_s": evals / (plain_ms * 1e-3),
            "speedup_vs_plain_per_box": plain_ms / batch_ms, "max_diff_over_tolerance": worst,
            "create_s": create_s, "tuning": tune, "context_cached_bytes_after": cached}


def cli_e2e(work: Path, evals: int):
    """The drop-in executable end to end on the same map set: `autogrid4_b200
    -p bench.gpf -l cli.glg` as a user runs it (process start, CUDA context,
    GPF and PDBQT parsing, tables, bond vectors, maps, map text formatted on
    the GPU, .map/.fld/.xyz files written).  Whole-process wall time, best of 2
    (the first run also pages the image in)."""
    cli = ROOT / "autogrid_b200" / "_build" / "autogrid4_b200"
    if not cli.exists():
        return None
    walls = []
    for _ in range(2):
        t0 = time.perf_counter()
        r = subprocess.run([str(cli), "-p", "bench.gpf", "-l", "cli.glg"], cwd=work, capture_output=True, text=True)
        walls.append(time.perf_counter() - t0)
        if r.returncode != 0:
            return {"error": r.stderr[-300:]}
    ok = "Successful Completion" in (work / "cli.glg").read_text()
    return {"command": "autogrid4_b200 -p bench.gpf -l cli.glg", "seconds": min(walls), "ok": ok,
            "evals_per_s": evals / min(walls),
            "note": "whole process, files written; compare the reference's whole-process wall in cpu_baseline"}


def batched_sharded(ctx, n, work: Path, stream, rank: int, world: int):
    """The batched ensemble split by instance over the ranks
    (shard.partition_instances, greedy by points x atoms): each rank runs its
    share as one batch; the ensemble's time is the slowest rank's (L2 flushed,
    CUDA events, mean of 5)."""
    import torch
    from autogrid_b200 import Batch, Job, synth
    from autogrid_b200.shard import instance_cost, partition_instances
    d = work / "ensemble"
    gpfs = synth.write_ensemble(d, n, seed=2024)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        probs = [Job(os.path.basename(g), None).problem() for g in gpfs]
    finally:
        os.chdir(cwd)
    share = partition_instances([instance_cost(p) for p in probs], world)[rank]
    mine = [probs[i] for i in share]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    b = Batch(ctx, mine) if mine else None
    vals = []
    if b is not None:
        b.run(stream.cuda_stream)
        torch.cuda.synchronize()
        for _ in range(5):
            flush.zero_()
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            b.run(stream.cuda_stream)
            e_.record(stream)
            torch.cuda.synchronize()
            vals.append(s_.elapsed_time(e_))
        b.close()
    ms = max_over_ranks([float(np.mean(vals)) if vals else 0.0], world, "cuda")[0]
    evals = sum(p.points * p.n_maps for p in probs)
    return {"instances": n, "split": f"by instance over {world} ranks (greedy, points x atoms)",
            "ms_per_ensemble": ms, "evals_per_s": evals / (ms * 1e-3) if ms else None}


def differentiable_maps(ctx, work: Path, stream, reps: int = 10):
    """The differentiable form: 4,000-atom receptor (same generator), npts
    60^3, 8 maps, linear-table mode.  Forward and adjoint device times of the
    FP32 kernels (ag_diff_timing events; L2 flushed before each), the
    end-to-end forward + backward through the torch.autograd binding, and the
    gradient checks of autogrid_b200.gradcheck on 64 random atoms for
    L = sum(w * maps), w ~ N(0, 1)."""
    import torch
    from autogrid_b200 import Diff, Job, gradcheck, synth
    from autogrid_b200.torch_maps import GridMaps
    d = work / "diff"
    rec = synth.make_receptor(4000, seed=7, center=(0.0, 0.0, 0.0))
    spec = synth.GridSpec(npts=(60, 60, 60))
    g = synth.write_case(d, "c3", rec, spec)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        job = Job(g.name, None)
    finally:
        os.chdir(cwd)
    prob = job.problem()
    P, M = prob.points, prob.n_maps
    rng = np.random.default_rng(0)
    w = rng.normal(size=prob.map_shape)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    df = Diff(ctx, prob, "fp32")
    w32 = w.astype(np.float32)
    df.forward()
    df.backward(w32)
    chs = []  # the closest-H search alone (runs when coordinates change), warm
    for _ in range(5):
        flush.zero_(); torch.cuda.synchronize()
        df.forward()
        chs.append(df.timing()[1])
    ch_ms = float(np.median(chs))
    fw, bw = [], []
    for _ in range(reps):
        flush.zero_(); torch.cuda.synchronize()
        df.forward(keep_closest_h=True)
        fw.append(df.timing()[0])
        flush.zero_(); torch.cuda.synchronize()
        df.backward(w32)
        bw.append(df.timing()[2])
    df.close()
    fwd_ms, bwd_ms = float(np.median(fw)), float(np.median(bw))
    # end to end through torch: host coordinates in, gradients out
    fn = GridMaps(job, device=torch.cuda.current_device(), precision="fp32")
    wt = torch.tensor(w32, device="cuda")
    coords0 = torch.tensor(prob.arrays["coord"].reshape(-1, 3))
    charges0 = torch.tensor(prob.arrays["charge"])
    e2e = []
    for k in range(reps + 1):
        c = coords0.clone().requires_grad_(True)
        q = charges0.clone().requires_grad_(True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        loss = (wt * fn(c, q)).sum()
        loss.backward()
        torch.cuda.synchronize()
        if k:
            e2e.append(time.perf_counter() - t0)
    atoms = rng.choice(prob.n_atoms, 64, replace=False)
    hs = (1e-3, 1e-5)
    chk = gradcheck.check(job, prob, ctx, atoms, w, h_coord=hs, kink_free=True)
    return {
        "workload": "diff_4000_61cube_8maps", "atoms": prob.n_atoms, "points": P, "maps": M,
        "tables": "linear interpolation between bins (AG_TABLE_LINEAR)", "dtype": "f32 (FP64 twin as error oracle)",
        "forward_ms": fwd_ms, "backward_ms": bwd_ms, "adjoint_over_forward": bwd_ms / fwd_ms,
        "closest_h_search_ms": ch_ms,
        "forward_evals_per_s": P * M / (fwd_ms * 1e-3),
        "e2e_torch_forward_backward_ms": float(np.median(e2e)) * 1e3,
        "gradcheck": {
            "atoms_checked": len(atoms), "loss": "sum(w * maps), w ~ N(0,1) seeded",
            "h_charge": chk["h_charge"], "h_coord": list(hs),
            "fp32_vs_fp64_adjoint_coord": chk["fp32_vs_fp64_coord"],
            "fp32_vs_fp64_adjoint_charge": chk["fp32_vs_fp64_charge"],
            "fp64_adjoint_vs_fd_charge": chk["fp64_vs_fd_charge"],
            "fp32_adjoint_vs_fd_charge": chk["fp32_vs_fd_charge"],
            "fp64_adjoint_vs_fd_coord": {str(h): chk["fp64_vs_fd_coord"][h] for h in hs},
            "fp32_adjoint_vs_fd_coord": {str(h): chk["fp32_vs_fd_coord"][h] for h in hs},
            # the loss restricted, per component, to the grid points at which it has no slope
            # kink along the stencil (autogrid_b200.gradcheck.kink_mask): adjoint vs central
            # differences of that loss
            "fd_kink_free_error": {str(h): chk["fd_kink_free_coord"][h] for h in hs},
            "fd_kinked_components": {str(h): chk["fd_kinked_components"][h] for h in hs},
            "fd_components": chk["fd_components"],
            "fd_masked_point_fraction": {str(h): chk["fd_masked_point_fraction"][h] for h in hs},
            "error_norm": "||a - b||_2 / ||b||_2 over the checked components",
            "seconds": chk["fd_seconds"],
        },
    }


def vina_conformers(ctx, work: Path, stream, K: int = 32, reps: int = 5):
    """Batched differentiable Vina maps: K conformers of an 8,000-atom receptor
    (same generator; base structure plus N(0, 0.3 A) jitter on every
    coordinate), npts 100^3, Vina tables of 8 ligand types, linear-table mode.
    Forward and adjoint each run as one launch over all K conformers with
    pair terms recomputed in the adjoint; device times from ag_diff_timing
    (L2 flushed before each), and an end-to-end figure through the C ABI:
    host coordinates of all conformers in, maps computed, dL/d(maps) resident
    on the device, dL/d(coordinates) back on the host."""
    import torch
    from autogrid_b200 import Diff, Job, synth
    d = work / "vina"
    rec = synth.make_receptor(8000, seed=11, center=(0.0, 0.0, 0.0))
    spec = synth.GridSpec(npts=(100, 100, 100), ligand_types=["A", "C", "F", "HD", "N", "NA", "OA", "SA"])
    g = synth.write_case(d, "c4", rec, spec)
    cwd = os.getcwd()
    os.chdir(d)
    try:
        job = Job(g.name, None)
    finally:
        os.chdir(cwd)
    vp = job.vina_problem()
    rng = np.random.default_rng(4)
    base = vp.arrays["coord"].reshape(-1, 3)
    confs = [base + rng.normal(0.0, 0.3, base.shape) for _ in range(K)]
    df = Diff(ctx, vp, "fp32", conformers=K)
    for k, c in enumerate(confs):
        df.set_atoms(c, conformer=k)
    df.forward()
    grad = torch.randn(df.shape, dtype=torch.float32, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    torch.cuda.synchronize()
    df.backward(device_ptr=grad.data_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    fw, bw = [], []
    for _ in range(reps):
        flush.zero_(); torch.cuda.synchronize()
        df.forward(keep_closest_h=True)
        fw.append(df.timing()[0])
        flush.zero_(); torch.cuda.synchronize()
        df.backward(device_ptr=grad.data_ptr())
        bw.append(df.timing()[2])
    e2e = []
    for _ in range(3):
        t0 = time.perf_counter()
        for k, c in enumerate(confs):
            df.set_atoms(c, conformer=k)
        df.forward(keep_closest_h=True)
        df.backward(device_ptr=grad.data_ptr())
        e2e.append(time.perf_counter() - t0)
    # the same with the coordinates updated on the device: one pinned host
    # array of all conformers in, cell lists rebuilt by kernels, dL/d(coord)
    # of all conformers back into a pinned host array
    host_c = torch.tensor(np.stack(confs), dtype=torch.float64).pin_memory()
    host_g = torch.empty((K, vp.n_atoms, 3), dtype=torch.float64).pin_memory()
    dev_c = torch.empty_like(host_c, device="cuda")
    dev_g = torch.empty_like(host_g, device="cuda")
    e2e_dev = []
    for it in range(4):
        t0 = time.perf_counter()
        dev_c.copy_(host_c, non_blocking=True)
        torch.cuda.synchronize()
        df.set_atoms_device(dev_c.data_ptr())
        df.forward(keep_closest_h=True)
        df.backward_device(grad.data_ptr(), dev_g.data_ptr(), None)
        host_g.copy_(dev_g)
        if it:
            e2e_dev.append(time.perf_counter() - t0)
    df.close()
    P, M = vp.points, vp.n_maps
    fwd_ms, bwd_ms = float(np.median(fw)), float(np.median(bw))
    return {"workload": "vina_32x8000_101cube_8maps", "conformers": K, "atoms": vp.n_atoms, "points": P,
            "maps": M, "tables": "Vina (main.cpp:2081-2126 as written), linear interpolation",
            "forward_ms": fwd_ms, "backward_ms": bwd_ms, "adjoint_over_forward": bwd_ms / fwd_ms,
            "forward_evals_per_s": K * P * M / (fwd_ms * 1e-3),
            "forward_backward_evals_per_s": K * P * M / ((fwd_ms + bwd_ms) * 1e-3),
            "e2e_forward_backward_ms": float(np.median(e2e)) * 1e3,
            "e2e_note": "host coordinates through ag_diff_set_conformer (host cell lists) per conformer",
            "e2e_device_update_ms": float(np.median(e2e_dev)) * 1e3,
            "e2e_device_update_note": "all conformers' coordinates H2D, ag_diff_set_atoms_device (cell lists "
                                      "on the device), forward, ag_diff_backward_device, dL/dcoord D2H",
            "launches": {"forward": 1, "backward": 1},
            "parity": "unpinned against the reference (its Vina path is compiled out); tables pinned to the "
                      "source as written, maps to the C oracle"}


def serial_kernel_ms(ctx, plan, stream, steps):
    """Device times of a serial plan's kernels (events recorded around their
    launches by the library), averaged over L2-flushed runs: the far-field
    kernel with its fix-up (far_ms), the fix-up alone, and the near-field
    kernels; plus the near pairs per run."""
    import torch
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    far, fix, near = [], [], []
    st = None
    for _ in range(max(3, min(steps, 10))):
        flush.zero_()
        plan.run(stream.cuda_stream)
        st = ctx.stats()
        far.append(st.far_ms)
        fix.append(st.fixup_ms)
        near.append(st.near_ms)
    return {"far_ms": float(np.mean(far)), "fixup_ms": float(np.mean(fix)), "near_ms": float(np.mean(near)),
            "near_pairs": int(st.near_pairs)}


def peak_rates(lib, device):
    import ctypes as C
    try:
        fn = lib.ag_diag_peak_rates
    except AttributeError:
        return None, None, None
    fn.restype = C.c_int
    fn.argtypes = [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    r, f, c = C.c_double(), C.c_double(), C.c_double()
    if fn(device, C.byref(r), C.byref(f), C.byref(c)) != 0:
        return None, None, None
    return r.value, f.value, c.value


def profile_traffic(kernel: str):
    p = ROOT / "profiles" / "ncu_traffic.json"
    if not p.exists():
        return None
    try:
        return json.loads(p.read_text()).get(kernel, {}).get("dram_bytes_per_launch")
    except (ValueError, OSError):
        return None


def run_reference(args, rank, world):
    """The reference's own CPU implementation (OpenMP build from its sources),
    rank 0 only, each step a bounded z-slab sample of the workload."""
    if rank != 0:
        return
    from oracle.oracle import REF_BIN
    if not REF_BIN.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/autogrid4 was not built"}))
        return
    from autogrid_b200 import synth
    rec, spec = synth.workload(args.workload, seed=0)
    work = Path(tempfile.mkdtemp(prefix="agb_ref_"))
    threads = min(32, os.cpu_count() or 1)
    for _ in range(args.warmup):
        reference_sample(rec, spec, work, 1, nxy=4)
    rates, secs = [], []
    desc = ""
    for _ in range(args.steps):
        res = reference_sample(rec, spec, work, threads, nxy=24)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference run failed"}))
            return
        rate, dt, P, M, desc = res
        rates.append(rate)
        secs.append(dt)
    v = float(np.mean(rates))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": float(np.mean(secs)) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded receptor, shapes of the plain large map set)",
            "config": {"workload": args.workload, "sample": desc},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": "reference", "sample": desc},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    shutil.rmtree(work, ignore_errors=True)


if __name__ == "__main__":
    main()
