#!/usr/bin/env python3
"""Benchmark of the SPEX polarisation hot path on B200: chi0 band-pair TFLOP/s.

Workload (one GPU): N_MB=1200 mixed-basis functions, 64 k points, 40 occupied x
400 unoccupied bands (P = 1,024,000 band pairs), 24 imaginary frequencies, 1% of
the pairs near-degenerate (|e_n'-e_n| < 1e-6 eV). One step is one full
accumulation chi0_IJ(w) = sum_p M_Ip w_p(w) M*_Jp for all 24 frequencies into the
packed Hermitian output, output zeroed first (as `susceptibility` does).

  value        TFLOP/s of the headline (split-precision) path, inputs resident in
               HBM; algorithmic flops 8*N^2*P*Nw (full complex Gram)
  fp64         the plain FP64 drop-in path on the same inputs
  e2e          the same metric through the host-pointer drop-in call
               (spx_chi0_accumulate): cprod from pinned host memory every step,
               susceph copied back every step
  roofline     dominant kernel (the band-pair accumulation): achieved vs measured peak
  cpu_baseline the oracle port of the reference loop on the host cores, bounded sample
  --impl reference  times the reference CPU loop (oracle port) alone, on a fixed sample
               of the same workload per step; it imports neither the product package
               nor its library (inputs from oracle/ and numpy).

Multi-GPU: the pair axis is sharded (the reference's Mblocks split over
(k, occ, unocc)); each rank accumulates its share and the packed output is
summed with one NCCL reduce to rank 0 (Mreduce analogue).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "chi0 band-pair TFLOP/s, split-precision vs FP64 on one B200 at <=1e-6 rel err"
UNIT = "TFLOP/s"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), "measured"
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for k, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(k)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def inputs_module():
    """project1_b200/inputs.py loaded on its own (numpy only): the CPU arms take the
    workload shapes and energies from it without importing the product package."""
    import importlib.util
    name = "spx_workload_inputs"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, ROOT / "project1_b200" / "inputs.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


class CpuSample:
    """The oracle's faithful reference loop (src/susceptibility.f:1182-1240, per-(i,j)
    ddot per frequency) over a fixed sample of the workload: every element i <= j < J
    of the first J columns, all frequencies, all pairs. J is sized so that one run
    takes about `budget_s` on `threads` host threads. M comes from the oracle's own
    generator (the same bits as the GPU library's), energies from numpy."""

    def __init__(self, w, budget_s: float, threads: int = 0):
        import oracle
        inp = inputs_module()
        self.w = w
        self.threads = threads or os.cpu_count() or 1
        d = inp.pair_ediff(w)
        om = inp.frequencies(w.nw)
        self.wt = oracle.weights(d, om, None, 1.0 / w.nk)
        probe = oracle.gen_cmatrix(w.seed, w.stream_id, w.npair, 2, 0, w.m_scale, self.threads)
        t0 = time.perf_counter()
        oracle.chi0(probe, self.wt, threads=min(self.threads, 3))
        per_elem = (time.perf_counter() - t0) / 3 * min(self.threads, 3)   # thread-seconds
        target = budget_s * self.threads / per_elem
        self.ncol = int(max(2, min(w.nbas, (np.sqrt(8 * target + 1) - 1) / 2)))
        self.m = oracle.gen_cmatrix(w.seed, w.stream_id, w.npair, self.ncol, 0, w.m_scale,
                                    self.threads)
        self.nel = self.ncol * (self.ncol + 1) // 2
        self.full = w.nbas * (w.nbas + 1) / 2

    def run(self) -> float:
        import oracle
        t0 = time.perf_counter()
        oracle.chi0(self.m, self.wt, threads=self.threads)
        return time.perf_counter() - t0

    def tflops(self, dt: float) -> float:
        """The headline metric on the sample: the workload's algorithmic flops per
        element (8 N^2 P Nw over the N(N+1)/2 computed elements) times the sample's
        elements, per second."""
        return self.w.flops * (self.nel / self.full) / dt / 1e12

    def describe(self, dt: float) -> str:
        return (f"faithful per-(i,j) ddot loop (src/susceptibility.f:1182-1240) over the {self.nel} "
                f"elements i<=j<{self.ncol} of all {self.w.nw} frequencies and all {self.w.npair} "
                f"pairs ({self.nel / self.full:.2%} of the {self.full:.0f} elements), {dt:.1f} s per run "
                f"on {self.threads} threads; inputs from the oracle's generator")


def cpu_baseline(w, budget_s: float = 15.0, threads: int = 0):
    """One timed run of the faithful loop on a sample sized to `budget_s`."""
    smp = CpuSample(w, budget_s, threads)
    dt = smp.run()
    return {"value": smp.tflops(dt), "unit": UNIT, "cores": smp.threads, "kind": "port",
            "sample": smp.describe(dt), "seconds_sample": dt,
            "seconds_full_estimate": dt * smp.full / smp.nel}


def run_reference(args):
    """--impl reference: the oracle port of the reference's CPU loop on all host threads,
    each step one run over the same fixed sample of the workload. Rank 0 alone runs."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    inp = inputs_module()
    w = workload_from_args(args, inp)
    smp = CpuSample(w, args.ref_budget)
    for _ in range(args.warmup):
        smp.run()
    times = [smp.run() for _ in range(args.steps)]
    rates = [smp.tflops(t) for t in times]
    v = statistics.median(rates)
    ms = 1e3 * statistics.mean(times)
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded Philox4x32-10 normals from the oracle's generator, uniform energies, "
                "Gauss-Legendre frequencies)",
        "config": bench_config(w, args.gpus),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": smp.threads, "kind": "port",
                         "sample": smp.describe(statistics.median(times))},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_definition": "one run of the reference loop over the fixed element sample; value is "
                           "its rate in the workload's algorithmic flops",
        "sample_fraction": smp.nel / smp.full,
        "full_workload_s_estimate": statistics.median(times) * smp.full / smp.nel,
        "rates_min_max": [min(rates), max(rates)],
    }))


def workload_from_args(args, inp=None):
    """The named workload, optionally shrunk (--kpts / --freqs) for profiling captures."""
    import dataclasses
    if inp is None:
        from project1_b200 import inputs as inp
    w = inp.CONFIGS[args.workload]
    if args.kpts or args.freqs:
        w = dataclasses.replace(w, name=w.name + "-small", nk=args.kpts or w.nk, nw=args.freqs or w.nw)
    return w


def workload_name(w):
    return (f"{w.name}: chi0 N_MB={w.nbas}, {w.nk} k x {w.nocc} occ x {w.nunocc} unocc "
            f"(P={w.npair}), {w.nw} imaginary frequencies"
            + (f", {w.degenerate_frac:.0%} degenerate pairs" if w.degenerate_frac else ""))


def bench_config(w, world: int) -> dict:
    """The `config` of both arms' lines (identical for the same workload and N)."""
    return {"workload": workload_name(w), "nbas": w.nbas, "npair": w.npair, "nw": w.nw,
            "parallelism": f"pairs sharded over {world} GPU(s)",
            "l2": "inputs larger than L2 (M = %.1f GB)" % (16 * w.nbas * w.npair / 1e9)}


def int8_ops(N: int, P: int, nw: int, variant: int, slab: int) -> float:
    """int8 ops the accumulation kernel issues for P pairs: 6 digit products per real MAC
    of each 128 x 128 real-stacked MMA tile (one CTA or the persistent kernel: the upper
    64-blocks; CTA pair: two tiles per pair item), over the slabs padded to 64 pairs, 2 ops
    per MAC."""
    nblk = (N + 63) // 64
    if variant == 5:
        # 64 x 80 complex tiles: 128 x 160 real MMA tiles, column blocks of 80
        tiles = upper_tiles(N, 5)
        ncols = 160
    else:
        tiles = nblk * (nblk + 1) // 2 if variant in (1, 3) else 2 * sum(bj // 2 + 1 for bj in range(nblk))
        ncols = 128
    pad = sum(((min(slab, P - s0) + 63) // 64) * 64 for s0 in range(0, P, slab))
    return 2.0 * 6 * 128 * ncols * tiles * pad * nw


def fp64_roofline(ctx, N: int, achieved: float) -> dict:
    """Roofline of the FP64 accumulation (DMMA) against this GPU's DMMA rate, measured
    here by the library's own in-register DMMA loop. The kernel computes only the upper
    64 x 64 tiles, so the rate the pipe executes is the algorithmic rate times the
    executed share of the full Gram."""
    peak = ctx.measure_dmma_peak()
    nblk = (N + 63) // 64
    share = nblk * (nblk + 1) / 2 * 64 * 64 / (N * N)
    return {"bound": "tensor (FP64 DMMA)", "achieved": achieved, "peak": peak, "unit": UNIT,
            "frac": achieved / peak, "executed_tflops": achieved * share, "executed_frac": achieved * share / peak,
            "executed_share_of_full_gram": share, "traffic": None,
            "peak_source": "measured: spx_measure_dmma_peak (mma.sync m16n8k8 f64 loop, CUDA events)"}


def upper_tiles(N: int, variant: int) -> int:
    """Upper-region tiles the accumulation kernel visits per frequency: 64 x 64 complex
    tiles, or 64 x 80 for variant 5 (column blocks of 80, row blocks of 64)."""
    nblk = (N + 63) // 64
    if variant == 5:
        return sum(min((bj * 80 + 79) // 64, nblk - 1) + 1 for bj in range(-(-N // 80)))
    return nblk * (nblk + 1) // 2


def measured_traffic(kernel: str, nbas: int, nw: int, slab: int, npair_step: int, tiles: int = 0):
    """DRAM bytes of the dominant kernel from the committed ncu capture, scaled to one
    launch (one slab of all frequencies) of this shape: the capture's bytes per pair,
    frequency and 64-block tile. None when no capture of `kernel` is recorded."""
    f = ROOT / "profiles" / "roofline_traffic.json"
    if not f.exists():
        return None
    try:
        rec = json.loads(f.read_text()).get(kernel)
    except Exception:
        return None
    if not rec:
        return None
    if "by_slab" in rec:
        # the capture whose slab is nearest this one (traffic per pair falls with the slab)
        key = min(rec["by_slab"], key=lambda k: abs(int(k) - slab))
        rec = dict(rec["by_slab"][key], captured_slab=int(key))
    nblk = (nbas + 63) // 64
    tiles = tiles or nblk * (nblk + 1) // 2
    per_launch = rec["bytes_per_pair_freq_tile"] * min(slab, npair_step) * nw * tiles
    out = {"bytes_per_launch": per_launch, "launches_per_step": -(-npair_step // slab),
           "source": rec["source"]}
    if "captured_slab" in rec:
        out["captured_slab"] = rec["captured_slab"]
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    import project1_b200 as spx
    from project1_b200 import inputs

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    from project1_b200.parallel import pair_shard, reduce_partial
    w = workload_from_args(args)
    # shard the pair axis: rank r owns a contiguous block of whole k points (Mblocks)
    P = w.npair
    p_lo, p_hi = pair_shard(P, world, rank, block=w.nocc * w.nunocc)
    Pr = p_hi - p_lo
    N, nw = w.nbas, w.nw
    npk = spx.npack(N)
    # a pinned slab travels in the tuning table, which names the variant too
    ctx = spx.Context(local, split_variant=0 if args.slab else args.variant)
    stream = torch.cuda.current_stream(dev)

    # inputs resident in HBM: M (N, P) column blocks generated on device, bit-identical
    # to the host stream; energies / frequencies from the seeded host generator
    M = torch.empty((N, Pr), dtype=torch.complex128, device=dev)
    full_rows = P
    # generate this rank's pair range: element (p, c) of the full matrix
    gen = torch.empty((1, full_rows), dtype=torch.complex128, device=dev) if world > 1 else None
    if world == 1:
        ctx.gen_cmatrix_dev(w.seed, w.stream_id, M, P, scale=w.m_scale, stream=stream.cuda_stream)
    else:
        for c in range(N):
            ctx.gen_cmatrix_dev(w.seed, w.stream_id, gen, P, col0=c, scale=w.m_scale, stream=stream.cuda_stream)
            M[c].copy_(gen[0, p_lo:p_hi])
        del gen
    ediff_h = inputs.pair_ediff(w)
    ediff = torch.from_numpy(ediff_h[p_lo:p_hi].copy()).to(dev)
    omega_h = inputs.frequencies(nw)
    omega = torch.from_numpy(omega_h).to(dev)
    out = torch.zeros((nw, npk), dtype=torch.complex128, device=dev)
    torch.cuda.synchronize()

    def step(precision):
        out.zero_()
        st = ctx.chi0_accumulate_dev(M, ediff, omega, out, scale_all=1.0 / w.nk, precision=precision,
                                     stream=stream.cuda_stream, stats=True)
        reduce_partial(out, dst=0)
        return st

    def timed(precision, warmup, steps, sampler=None):
        for _ in range(warmup):
            step(precision)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        if sampler:
            sampler.start()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        gram_ms = []
        launches = 0
        for _ in range(steps):
            st = step(precision)
            gram_ms.append(st["ms_gram"])
            launches += st["kernel_launches"]
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        ms = e0.elapsed_time(e1) / steps
        if world > 1:
            t = torch.tensor([ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms, gram_ms, launches, clocks

    avail = {"split": True}
    if args.precision != "fp64":
        try:
            step("split")
            torch.cuda.synchronize()
        except spx.SpexGpuError as e:
            avail["split"] = False
            avail["split_error"] = str(e)
    head = "split" if avail["split"] else "fp64"
    if args.precision:
        head = args.precision

    # the autotuner picks the accumulation kernel and slab for this shape (untimed);
    # --slab pins one (profiling) through a one-entry tuning table
    tuned = None
    if head == "split" and args.slab:
        import tempfile
        tuned = {"variant": args.variant or 1, "slab_pairs": args.slab, "tflops": 0.0}
        entry = {"nbas_bucket": (N + 127) // 128, "npair_bucket": 0 if Pr <= 16384 else (1 if Pr <= 32768 else 2),
                 "nw": nw, "variant": tuned["variant"], "slab_pairs": args.slab,
                 "tile": 80 + 3 * 256 if tuned["variant"] == 3 else 0, "tflops": 0.0}
        with tempfile.TemporaryDirectory() as td:
            with open(os.path.join(td, "tune.json"), "w") as fh:
                json.dump({"format": "spexgpu-tune-1", "entries": [entry]}, fh)
            ctx.tune_load(os.path.join(td, "tune.json"))
    elif head == "split" and args.autotune:
        tuned = ctx.autotune_split(N, Pr, nw)
    sampler = ClockSampler(local) if rank == 0 else None
    ms, gram_ms, launches, clocks = timed(head, args.warmup, args.steps, sampler)
    value = w.flops / (ms * 1e-3) / 1e12   # whole job: all ranks' pairs / max-over-ranks time
    # FP64 drop-in on the same inputs (secondary line; same kernel every step, 1 warm-up)
    fp64 = None
    if head == "split" and args.fp64_steps > 0:
        ms64, gram64, _, _ = timed("fp64", 1, args.fp64_steps)
        fp64 = {"value": w.flops / (ms64 * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms64,
                "steps": args.fp64_steps, "warmup": 1, "kernel_ms": statistics.median(gram64)}

    # e2e through the host-pointer drop-in call, cprod in pinned host memory
    e2e = None
    if args.e2e_steps > 0:
        host = torch.empty((N, Pr), dtype=torch.complex128, pin_memory=True)
        host.copy_(M)
        out_h = np.zeros((npk, nw), dtype=np.complex128, order="F")
        eh = ediff_h[p_lo:p_hi].copy()
        ctx2 = spx.Context(local)
        if tuned is not None:
            # the tuning table travels as its JSON file
            import tempfile
            with tempfile.TemporaryDirectory() as td:
                ctx.tune_save(os.path.join(td, "tune.json"))
                ctx2.tune_load(os.path.join(td, "tune.json"))
        h2d = d2h = 0
        dt = 0.0
        for it in range(1 + args.e2e_steps):
            # the caller's output starts at zero each step (the reference zeroes susceph
            # before its packet loop); the timed region is the call itself, which
            # returns with the result in host memory
            out_h[:] = 0
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            t0 = time.perf_counter()
            st = ctx2.chi0_accumulate_host_ptr(host.data_ptr(), Pr, Pr, N, eh, omega_h, out_h,
                                               scale_all=1.0 / w.nk, precision=head)
            if it >= 1:
                dt += time.perf_counter() - t0
                h2d, d2h = st["h2d_bytes"], st["d2h_bytes"]
                e2e_dev = (st["ms_gram"], st["ms_prep"])
        dt /= args.e2e_steps
        if world > 1:
            t = torch.tensor([dt], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = float(t.item())
        e2e = {"value": w.flops / dt / 1e12, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": dt * 1e3, "steps": args.e2e_steps,
               "warmup": 1, "source": "pinned host memory; the caller zeroes its output before each call (untimed)"}
        # the host link's own rate (one pinned 2 GiB copy to the device, CUDA events): the
        # end-to-end step cannot beat its bytes over this rate
        nbw = min(host.numel(), (2 << 30) // 16)
        src = host.view(-1)[:nbw]
        dst = torch.empty(nbw, dtype=torch.complex128, device=dev)
        dst.copy_(src, non_blocking=True)
        torch.cuda.synchronize()
        c0 = torch.cuda.Event(enable_timing=True)
        c1 = torch.cuda.Event(enable_timing=True)
        c0.record()
        dst.copy_(src, non_blocking=True)
        c1.record()
        torch.cuda.synchronize()
        h2d_gbs = 16.0 * nbw / (c0.elapsed_time(c1) * 1e-3) / 1e9
        del dst
        e2e["h2d_link_gbs"] = h2d_gbs
        # device time inside the call (accumulation kernels; preparation the compute
        # stream waited for), the rest waits for the host copies
        e2e["accumulation_ms"], e2e["preparation_ms"] = e2e_dev
        e2e["copy_bound_ms"] = (h2d + d2h) / (h2d_gbs * 1e9) * 1e3
        e2e["roofline"] = {"bound": "host link (PCIe)", "achieved_gbs": (h2d + d2h) / dt / 1e9,
                           "peak_gbs": h2d_gbs, "frac": (h2d + d2h) / dt / 1e9 / h2d_gbs,
                           "peak_source": "measured: one 2 GiB pinned host-to-device copy"}
        ctx2.close()
        del host

    # accuracy of the headline path vs the FP64 path, all elements (and FP64 vs oracle samples)
    acc = None
    if rank == 0 and world == 1 and head == "split" and args.check:
        acc = accuracy_check(ctx, w, M, ediff, omega, stream, ediff_h, omega_h)

    hbm, bf16, bf16s, src = peaks()
    kernel_ms = statistics.median(gram_ms)
    # the dominant kernel per step is the accumulation over all 24 frequencies: algorithmic
    # flops 8 N^2 P Nw per step (per rank: its own pairs)
    ach = w.flops * (Pr / P) / (kernel_ms * 1e-3) / 1e12
    if head == "split":
        roof = {"bound": "tensor", "achieved": ach, "peak": bf16s, "unit": UNIT, "frac": ach / bf16s,
                "traffic": None, "peak_source": f"{src} bf16_tflops_sustained (kernel timed inside a long step)"}
        # the same kernel seen from the int8 pipe it runs on, for the variant and slab that ran
        variant = tuned["variant"] if tuned else (ctx.split_variant if ctx.split_variant in (1, 3, 5) else 2)
        slab = tuned["slab_pairs"] if tuned else 32768
        ops = int8_ops(N, Pr, nw, variant, slab)
        i8 = ops / (kernel_ms * 1e-3) / 1e12
        roof["int8_pipe"] = {"int8_ops_per_step": ops, "variant": variant, "slab_pairs": slab,
                             "achieved_tops": i8, "peak_tops": 2 * bf16s, "frac": i8 / (2 * bf16s),
                             "peak_source": "2 x measured bf16 sustained (int8 peak is 16384 ops/cycle/SM "
                                            "in ncu, twice the bf16 pipe)"}
        kname = {1: "split_gram_kernel", 2: "split_gram2_kernel", 3: "pb_kernel",
                 5: "split_gram_kernel_64x80"}.get(variant, "split_gram_kernel")
        tr = measured_traffic(kname, N, nw, slab, Pr, upper_tiles(N, variant))
        if tr:
            nblk = (N + 63) // 64
            R = ((nblk + 1) // 2 * 2 if variant == 2 else nblk) * 128   # plane rows (the pair needs even blocks)
            roof["traffic"] = tr["bytes_per_launch"]
            roof["traffic_detail"] = dict(tr, kernel=kname, unit="bytes per launch (one slab, all frequencies)",
                                          operand_plane_bytes_per_launch=3.0 * nw * R * min(slab, Pr))
    else:
        roof = fp64_roofline(ctx, N, ach)
    if fp64 is not None:
        fp64["roofline"] = fp64_roofline(ctx, N, w.flops * (Pr / P) / (fp64["kernel_ms"] * 1e-3) / 1e12)

    if rank == 0:
        res = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None,
            "dtype": "int8 (3-digit slices of sqrt|w| M, 6 products)->int32->f64" if head == "split" else "f64",
            "data": "synthetic (seeded Philox4x32-10 normals, uniform energies, Gauss-Legendre frequencies)",
            "config": bench_config(w, world),
            "headline_precision": head,
            "autotuned": None if tuned is None else {k: tuned[k] for k in ("variant", "slab_pairs", "tflops")},
            "fp64": fp64, "e2e": e2e, "roofline": roof, "clocks": clocks,
            "gpu_launches": launches, "kernel_ms_per_step": kernel_ms,
            "flops_per_step": w.flops, "flops_hermitian_per_step": w.flops_hermitian,
            "accuracy": acc, "split_available": avail,
        }
        if fp64:
            res["speedup_vs_fp64"] = value / fp64["value"]
        if world == 1 and args.cpu_budget > 0:
            res["cpu_baseline"] = cpu_baseline(w, budget_s=args.cpu_budget)
    ctx.close()
    del M
    if rank == 0 and world == 1:
        torch.cuda.empty_cache()
        if args.products_steps > 0:
            res["c4_products_chi0"] = bench_products(args, dev, stream)
            torch.cuda.empty_cache()
        if args.batched_steps > 0:
            res["c3_batched"] = bench_batched(args, dev, stream)
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        dist.destroy_process_group()


def bench_batched(args, dev, stream):
    """Batched workload: 32 uneven q points, M generated on the device slab by slab, all q in
    one persistent kernel per step (tile shape and slab autotuned per (N, P) bucket in the
    warm-up)."""
    import torch
    import project1_b200 as spx
    from project1_b200 import _lib, inputs
    bw = inputs.BATCHED_CONFIGS["c3"]
    if args.c3_kpts:
        import dataclasses
        bw = dataclasses.replace(bw, nk=args.c3_kpts)
    qws = inputs.batched_qs(bw)
    if args.c3_qs:
        qws = qws[:args.c3_qs]
    omega = torch.from_numpy(inputs.frequencies(bw.nw)).to(dev)
    ctx = spx.Context(dev.index or 0)
    qs = []
    for qw in qws:
        qs.append(dict(nbas=qw.nbas, npair=qw.npair, seed=qw.seed, stream_id=qw.stream_id,
                       m_scale=qw.m_scale, ediff=torch.from_numpy(inputs.pair_ediff(qw)).to(dev),
                       scale_all=1.0 / qw.nk,
                       susceph=torch.zeros((bw.nw, spx.npack(qw.nbas)), dtype=torch.complex128,
                                           device=dev)))
    flops = sum(q.flops for q in qws)
    # role cycle counters of the persistent kernel (captured with the graph)
    ctx.pb_profile_enable(True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(args.batched_warmup):
        for q in qs:
            q["susceph"].zero_()
        ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_AUTOTUNE if i == 0 and args.autotune else 0,
                         stream=stream.cuda_stream, stats=True)
    warm_s = time.perf_counter() - t0
    ctx.pb_profile_enable(True)   # zeroed: the timed batches only
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    kernels = 0
    sampler = ClockSampler(dev.index or 0)
    sampler.start()
    e0.record(stream)
    for _ in range(args.batched_steps):
        for q in qs:
            q["susceph"].zero_()
        st = ctx.chi0_batched(qs, omega, stream=stream.cuda_stream, stats=True)
        kernels = st["kernel_launches"]
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.batched_steps
    prof = ctx.pb_profile_read()
    ctx.pb_profile_enable(False)
    cta = prof.pop("cta") or 1.0
    role = {k: round(v / cta, 4) for k, v in prof.items() if not k.endswith("_items")}
    role.update({k: int(v) for k, v in prof.items() if k.endswith("_items")})
    tune = [ctx.tune_lookup_batched(q["nbas"], q["npair"], bw.nw) for q in qs]
    # accuracy at full size on three q (the two cheapest and the median by flops):
    # the same batched call in FP64 against the split result of the timed batch
    acc = None
    if args.check:
        order = sorted(range(len(qws)), key=lambda k: qws[k].flops)
        pick = sorted({order[0], order[1], order[len(order) // 2]})
        sub = [dict(qs[k], susceph=torch.zeros_like(qs[k]["susceph"])) for k in pick]
        ctx.chi0_batched(sub, omega, precision="fp64", stream=stream.cuda_stream)
        torch.cuda.synchronize()
        per_q = [dict(compare_packed(qs[k]["susceph"], sq["susceph"], qws[k].nbas), q=k,
                      nbas=qws[k].nbas, npair=qws[k].npair) for k, sq in zip(pick, sub)]
        acc = {"split_vs_fp64_per_q": per_q,
               "max_normalized": max(x["max_normalized"] for x in per_q),
               "raw_rel_max": max(x["raw_rel_max"] for x in per_q)}
        del sub
    # the same batch as per-slab kernels (generation, quantizer, one-CTA accumulation)
    # replayed from one graph: the schedule the persistent kernel replaces, for comparison
    for q in qs:
        q["susceph"].zero_()
    ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_KERNELS | (_lib.SPX_BATCH_AUTOTUNE if args.autotune else 0),
                     stream=stream.cuda_stream)
    for q in qs:
        q["susceph"].zero_()
    e0.record(stream)
    stk = ctx.chi0_batched(qs, omega, flags=_lib.SPX_BATCH_KERNELS, stream=stream.cuda_stream, stats=True)
    e1.record(stream)
    torch.cuda.synchronize()
    ms_k = e0.elapsed_time(e1)
    slab_kernels = {"value": flops / (ms_k * 1e-3) / 1e12, "ms_per_step": ms_k,
                    "kernels_per_step": stk["kernel_launches"],
                    "note": "SPX_BATCH_KERNELS: the per-slab kernels of the single call in one graph"}
    res = {"workload": f"c3: {len(qws)} q, N_MB U{{{bw.nbas_range[0]}..{bw.nbas_range[1]}}}, "
                       f"occ U{{{bw.occ_range[0]}..{bw.occ_range[1]}}} x unocc "
                       f"U{{{bw.unocc_range[0]}..{bw.unocc_range[1]}}}, {bw.nk} k, {bw.nw} freqs, split",
           "value": flops / (ms * 1e-3) / 1e12, "unit": UNIT, "ms_per_step": ms,
           "steps": args.batched_steps, "warmup": args.batched_warmup,
           "warmup_s_incl_autotune_and_capture": warm_s, "flops_per_step": flops,
           "npair_total": sum(q.npair for q in qws), "graph_launches_per_step": 1,
           "kernels_per_step": kernels,
           "tuned_choices": sorted({(t["nbas_bucket"], t["npair_bucket"], "tile %dx%d, %d stages" % (
                                        64, t["tile"] & 255, t["tile"] >> 8), t["slab_pairs"])
                                    for t in tune if t}),
           "schedule": "one persistent kernel per batch (accumulation and operand-preparation "
                       "queues on every SM), captured in a CUDA graph",
           "m_generated_on_device": True, "clocks": clocks, "slab_kernels": slab_kernels,
           "role_profile": dict(role, note="cycles of one thread per role and CTA as a fraction of the "
                                           "CTAs' cycles (spx_pb_profile_read), summed over the timed batches"),
           "accuracy": acc}
    ctx.close()
    return res


def bench_products(args, dev, stream):
    """Products workload: wave-function products (MT Gaunt contraction + interstitial
    convolution) and split chi0 in one call, M never leaving the device."""
    import torch
    import project1_b200 as spx
    from project1_b200 import _lib, inputs
    from project1_b200.wavefproducts import (MtDesc, PwDesc, chi0_from_coeffs, wavefproducts2_mt,
                                             wavefproducts2_pw)
    w = inputs.WFPROD_CONFIGS["c4"]
    if args.c4_kpts:
        import dataclasses
        w = dataclasses.replace(w, nk=args.c4_kpts)
    mt, pw = MtDesc(inputs.mt_basis(w)), PwDesc(inputs.pw_basis(w))
    m1, m2 = inputs.mt_coeffs(w)
    p1, p2 = inputs.pw_coeffs(w, {"gpt1": pw.gpt1, "gpt2": pw.gpt2})
    D = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    m1, m2, p1, p2 = D(m1), D(m2), D(p1), D(p2)
    ew = inputs.Chi0Workload("c4", w.nbas, w.nk, w.nocc, w.nunocc, w.nw, seed=w.seed)
    ediff = D(inputs.pair_ediff(ew))
    omega = D(inputs.frequencies(w.nw))
    out = torch.zeros((w.nw, spx.npack(w.nbas)), dtype=torch.complex128, device=dev)
    ctx = spx.Context(dev.index or 0)
    sc = stream.cuda_stream
    # the accumulation kernel and slab for the chi0 part of this shape (untimed)
    tuned4 = ctx.autotune_split(w.nbas, w.npair, w.nw) if args.autotune else None

    def timed(fn, warmup, steps):
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

    def fused():
        out.zero_()
        chi0_from_coeffs(ctx, mt, pw, m1, m2, p1, p2, ediff, omega, out, scale_all=1.0 / w.nk,
                         precision="split", stream=sc)
    ms = timed(fused, args.products_warmup, args.products_steps)
    out.zero_()
    st = chi0_from_coeffs(ctx, mt, pw, m1, m2, p1, p2, ediff, omega, out, scale_all=1.0 / w.nk,
                          precision="split", stream=sc, stats=True)
    # accuracy at full size: the same call in FP64 (products and chi0) on every element,
    # and sampled elements against the oracle from the FP64 products' columns
    acc = None
    if args.check:
        out64 = torch.zeros_like(out)
        chi0_from_coeffs(ctx, mt, pw, m1, m2, p1, p2, ediff, omega, out64, scale_all=1.0 / w.nk,
                         precision="fp64", stream=sc)
        torch.cuda.synchronize()
        acc = {"split_vs_fp64": compare_packed(out, out64, w.nbas)}
    cp = torch.zeros((w.nbas, w.npair), dtype=torch.complex128, device=dev)
    if args.check:
        import oracle
        ctx64 = spx.Context(dev.index or 0, products=_lib.SPX_PRODUCTS_FP64)
        wavefproducts2_mt(ctx64, mt, m1, m2, cp, stream=sc)
        wavefproducts2_pw(ctx64, pw, p1, p2, cp, w.nbasp, stream=sc)
        torch.cuda.synchronize()
        ctx64.close()
        rng = np.random.default_rng(6)
        cols = sorted(set(rng.integers(0, w.nbas, 16).tolist()) | {0, w.nbasp - 1, w.nbasp, w.nbas - 1})
        colv = {c: cp[c].cpu().numpy() for c in cols}
        wt = oracle.weights(inputs.pair_ediff(ew), inputs.frequencies(w.nw), None, 1.0 / w.nk)
        acc.update(oracle_samples(out, out64, cols, colv, wt))
        acc["oracle_columns_from"] = "FP64 device products (the split call's products are int8 slices)"
        del out64
        cp.zero_()
    mt_ms = timed(lambda: wavefproducts2_mt(ctx, mt, m1, m2, cp, stream=sc), 1, 2)
    pw_ms = timed(lambda: wavefproducts2_pw(ctx, pw, p1, p2, cp, w.nbasp, stream=sc), 1, 2)
    ctx_s = spx.Context(dev.index or 0, products=_lib.SPX_PRODUCTS_SPLIT)
    pws_ms = timed(lambda: wavefproducts2_pw(ctx_s, pw, p1, p2, cp, w.nbasp, stream=sc), 1, 2)
    ctx_s.close()
    pwf = PwDesc(dict(inputs.pw_basis(w), nfft=48))
    pwf_ms = timed(lambda: wavefproducts2_pw(ctx, pwf, p1, p2, cp, w.nbasp, stream=sc), 1, 2)
    fl_mt = 8.0 * w.nunocc * w.maxlm * w.nocc * w.maxllm * w.nk * w.natom
    fl_pw = 8.0 * w.nunocc * w.ngpt * w.nocc * w.ngptm * w.nk
    res = {"workload": f"c4: {w.natom} atoms lmax {w.lcut} x {w.nrad} radial (maxlm {w.maxlm}), "
                       f"{w.ngpt} PW, {w.ngptm} MPB PW, N_MB {w.nbas}, {w.nk} k, {w.nocc} x {w.nunocc} "
                       f"bands, {w.nw} freqs; chi0 split, interstitial product GEMM on int8 "
                       f"slices (MT and convolution FP64)",
           "value": w.flops / (ms * 1e-3) / 1e12, "unit": UNIT + " (chi0 flops over products + chi0 time)",
           "ms_per_step": ms, "steps": args.products_steps, "warmup": args.products_warmup,
           "chi0_kernel_ms": st["ms_gram"], "products_and_prep_ms": st["ms_prep"],
           "mt_ms": mt_ms, "mt_tflops_fp64": fl_mt / (mt_ms * 1e-3) / 1e12,
           "pw_ms": pw_ms, "pw_tflops_fp64": fl_pw / (pw_ms * 1e-3) / 1e12,
           "pw_split_ms": pws_ms, "pw_split_tflops_equiv": fl_pw / (pws_ms * 1e-3) / 1e12,
           "pw_fft_branch_ms": pwf_ms, "pw_fft_grid": 48,
           "kernels_per_step": st["kernel_launches"], "m_bytes_on_device": 16 * w.nbas * w.npair,
           "chi0_autotuned": None if tuned4 is None else {k: tuned4[k] for k in ("variant", "slab_pairs", "tflops")},
           "accuracy": acc}
    # rooflines of the products: the GEMMs against the tensor pipes they run on, and
    # the HBM bytes the products must move (the M columns they write) against the
    # measured copy bandwidth
    hbm, _, bf16s, src = peaks()
    dmma = ctx.measure_dmma_peak()
    mt_pad = -(-w.nunocc // 64) * 64
    i8_pw = 2.0 * 9 * 4 * mt_pad * w.nocc * w.ngptm * (-(-w.ngpt // 64) * 64) * w.nk
    m_bytes = 16.0 * w.npair * w.nbas
    res["products_roofline"] = {
        "mt_gemm": {"bound": "tensor (FP64 DMMA)", "achieved_tflops": fl_mt / (mt_ms * 1e-3) / 1e12,
                    "peak_tflops": dmma, "frac": fl_mt / (mt_ms * 1e-3) / 1e12 / dmma,
                    "peak_source": "measured: spx_measure_dmma_peak"},
        "pw_gemm_int8": {"bound": "tensor (int8)", "int8_ops": i8_pw, "achieved_tops": i8_pw / (pws_ms * 1e-3) / 1e12,
                         "peak_tops": 2 * bf16s, "frac": i8_pw / (pws_ms * 1e-3) / 1e12 / (2 * bf16s),
                         "peak_source": f"2 x {src} bf16_tflops_sustained"},
        "hbm": {"bound": "hbm", "algorithmic_bytes": m_bytes, "ms": mt_ms + pws_ms,
                "achieved_gbs": m_bytes / ((mt_ms + pws_ms) * 1e-3) / 1e9, "peak_gbs": hbm,
                "frac": m_bytes / ((mt_ms + pws_ms) * 1e-3) / 1e9 / hbm,
                "note": "the products write the M columns once (MT then PW); neither kernel is HBM-bound "
                        "(ncu per-kernel DRAM figures are committed beside the profiles)"},
    }
    ctx.close()
    return res


def compare_packed(a, b, N: int) -> dict:
    """Errors of the packed output `a` (split) against `b` (FP64) on every element:
    normalised |d chi_ij| / sqrt(|chi_ii chi_jj|) (the metric the <= 1e-6 claim uses:
    every imaginary-axis weight has one sign, so |chi_ij| <= sqrt(chi_ii chi_jj)),
    raw |d chi_ij| / |chi_ij|, and Frobenius."""
    import torch
    j = torch.arange(N, device=a.device)
    d = b[:, j * (j + 1) // 2 + j].real.abs()                  # (nw, N)
    iu = torch.triu_indices(N, N, device=a.device)
    idx = iu[1] * (iu[1] + 1) // 2 + iu[0]
    diff = (a[:, idx] - b[:, idx]).abs()
    err = diff / torch.sqrt(d[:, iu[0]] * d[:, iu[1]])
    raw = diff / b[:, idx].abs().clamp_min(1e-300)
    sub = raw.flatten()[:: max(1, raw.numel() // 4000000)]
    return {"max_normalized": float(err.max()),
            "frac_normalized_above_1e-6": float((err > 1e-6).double().mean()),
            "frobenius": float(torch.linalg.norm(a - b) / torch.linalg.norm(b)),
            "raw_rel_max": float(raw.max()),
            "raw_rel_median": float(raw.median()),
            "raw_rel_p99": float(torch.quantile(sub, 0.99)),
            "frac_raw_above_1e-6": float((raw > 1e-6).double().mean()),
            "elements": int(err.numel()),
            "claim_metric": "max_normalized (|d chi_ij| / sqrt(|chi_ii chi_jj|), every element and "
                            "frequency); raw per-element relative error is unbounded where an "
                            "off-diagonal chi_ij nearly cancels"}


def oracle_samples(a, b, cols, colv, wt) -> dict:
    """Sampled elements (i, j) of consecutive sampled columns against the oracle's
    extended-precision element, normalised by its own diagonal."""
    ah, bh = a.cpu().numpy(), b.cpu().numpy()
    import oracle
    e64 = es = 0.0
    for k in range(len(cols) - 1):
        i, jj = cols[k], cols[k + 1]
        ref = oracle.chi0_element(colv[i], colv[jj], wt)
        refi = oracle.chi0_element(colv[i], colv[i], wt).real
        refj = oracle.chi0_element(colv[jj], colv[jj], wt).real
        sc = np.sqrt(np.abs(refi * refj))
        p = jj * (jj + 1) // 2 + i
        e64 = max(e64, float(np.max(np.abs(bh[:, p] - ref) / sc)))
        es = max(es, float(np.max(np.abs(ah[:, p] - ref) / sc)))
    return {"fp64_vs_oracle_sampled_max_normalized": e64,
            "split_vs_oracle_sampled_max_normalized": es, "oracle_samples": len(cols) - 1}


def accuracy_check(ctx, w, M, ediff, omega, stream, ediff_h, omega_h, nsample=24):
    """Split vs FP64 on every element; both vs the extended-precision oracle on sampled
    elements (columns regenerated by the oracle's own generator, the same bits)."""
    import torch

    import oracle
    import project1_b200 as spx
    N, nw = w.nbas, w.nw
    outs = {}
    for prec in ("split", "fp64"):
        o = torch.zeros((nw, spx.npack(N)), dtype=torch.complex128, device=M.device)
        ctx.chi0_accumulate_dev(M, ediff, omega, o, scale_all=1.0 / w.nk, precision=prec,
                                stream=stream.cuda_stream)
        outs[prec] = o
    torch.cuda.synchronize()
    a, b = outs["split"], outs["fp64"]
    res = {"split_vs_fp64": compare_packed(a, b, N)}
    rng = np.random.default_rng(5)
    wt = oracle.weights(ediff_h, omega_h, None, 1.0 / w.nk)
    cols = sorted(set(rng.integers(0, N, nsample).tolist()) | {0, N - 1})
    colv = {c: oracle.gen_cmatrix(w.seed, w.stream_id, w.npair, 1, c, w.m_scale)[:, 0] for c in cols}
    res.update(oracle_samples(a, b, cols, colv, wt))
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c0", "c1", "c2"])
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--ref-budget", type=float, default=10.0)
    ap.add_argument("--no-check", dest="check", action="store_false")
    ap.add_argument("--no-autotune", dest="autotune", action="store_false",
                    help="keep the default accumulation kernel instead of the tuned one")
    ap.add_argument("--products-steps", type=int, default=3, help="timed steps of the fused products workload (0: skip)")
    ap.add_argument("--products-warmup", type=int, default=3)
    ap.add_argument("--batched-steps", type=int, default=1, help="timed batches of the batched q-point workload (0: skip)")
    ap.add_argument("--batched-warmup", type=int, default=1)
    ap.add_argument("--c4-kpts", type=int, default=0, help="override the products workload's k-point count (profiling)")
    ap.add_argument("--c3-kpts", type=int, default=0, help="override the batched workload's k-point count (profiling)")
    ap.add_argument("--c3-qs", type=int, default=0, help="only the first n q points of the batched workload (profiling)")
    ap.add_argument("--precision", choices=["split", "fp64"], default=None,
                    help="force the measured path (profiling captures)")
    ap.add_argument("--variant", type=int, default=0, choices=[0, 1, 2, 3, 5],
                    help="accumulation kernel: 1 one CTA per 64 x 64 tile, 2 CTA pair, 3 persistent "
                         "schedule, 5 one CTA per 64 x 80 tile, 0 the library's choice")
    ap.add_argument("--slab", type=int, default=0,
                    help="pin the split path's slab (pairs per exact accumulation; profiling)")
    ap.add_argument("--kpts", type=int, default=0, help="override the k-point count (profiling)")
    ap.add_argument("--freqs", type=int, default=0, help="override the frequency count (profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
