#!/usr/bin/env python
"""Benchmark of the trace commitment: committed trace cells/sec.

Default workload (one step = one pcs.commit of the whole batch): the batched,
uneven KoalaBear shard -- 32 traces with log2 heights uniform on 10..22 and
widths uniform on 8..400, rescaled to 2^30 +- 3% trace cells, log_blowup 1,
one MMCS commit over all heights (rows of shorter matrices injected at their
level).  Inputs are seeded synthetic field elements (uniform in [0, p)); the
reference publishes no dataset for this path.

value  : cells / s with the traces already resident in HBM (device inputs);
e2e    : the same commit through the C ABI from pinned host buffers, the
         host -> device copies and the root read-back inside the timed region;
timing : CUDA events bracketing the K steps (after barrier + synchronize),
         max over ranks; inputs (4 GiB) exceed L2, so no flush is needed.

--gpus N runs N independent replicas (one process per GPU, launched by
torchrun): each rank commits its own shard, no data-path collective (weak
scaling).  --impl reference times the CPU oracle (the restated reference
algorithm, C + OpenMP) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "committed trace cells/sec (LDE+Poseidon2 Merkle, bit-exact roots)"
UNIT = "cells/s"


# ---------------------------------------------------------------- workloads
def uneven_kb_shapes(seed: int = 2, n: int = 32, target_log: int = 30, lo: int = 10, hi: int = 22):
    """32 (log_height, width) pairs: log heights uniform on [lo, hi], widths
    uniform on [8, 400], widths rescaled so the cells land within 3% of 2^30."""
    target = 1 << target_log
    for attempt in range(1000):
        rng = np.random.default_rng(seed * 1000 + attempt)
        logh = rng.integers(lo, hi + 1, size=n)
        w = rng.integers(8, 401, size=n).astype(np.float64)
        cells = float((w * (2.0 ** logh)).sum())
        w2 = np.clip(np.round(w * target / cells), 8, 400).astype(np.int64)
        tot = int((w2 << logh).sum())
        if abs(tot / target - 1) < 0.03:
            return [(int(a), int(b)) for a, b in zip(logh, w2)]
    raise RuntimeError("could not draw the workload")


def recursion_bb_shapes(seed: int = 3, n: int = 48, lo: int = 8, hi: int = 20):
    """48 BabyBear traces: log2 heights uniform on [8, 20], widths uniform on [4, 600]."""
    rng = np.random.default_rng(seed)
    logh = rng.integers(lo, hi + 1, size=n)
    w = rng.integers(4, 601, size=n)
    return [(int(a), int(b)) for a, b in zip(logh, w)]


WORKLOADS = {
    "uneven-kb-2^30": dict(field=0, log_blowup=1, shapes=lambda: uneven_kb_shapes(), seed=2),
    "recursion-bb-48": dict(field=1, log_blowup=2, shapes=lambda: recursion_bb_shapes(), seed=3),
    "single-kb-2^16x64": dict(field=0, log_blowup=1, shapes=lambda: [(16, 64)], seed=1),
    # same shape distribution scaled to 2^25 cells (heights 2^6..2^18): for profiler captures
    "uneven-kb-2^25": dict(field=0, log_blowup=1, shapes=lambda: uneven_kb_shapes(target_log=25, lo=6, hi=18),
                           seed=2),
    # one tall narrow trace (2^11-point sub-transforms, ~2 GB on the device): for profiler captures
    "single-kb-2^22x16": dict(field=0, log_blowup=1, shapes=lambda: [(22, 16)], seed=4),
}


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout: float = 5.0):
        """Block until nvidia-smi has printed its first sample, so that a timed
        region shorter than its start-up still has samples around it."""
        t0 = time.time()
        while self.proc and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.005)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


# Algorithmic Poseidon2 work: modular multiplications per permutation (S-box
# products plus one internal-diagonal product per lane per partial round;
# additions excluded): KoalaBear 8*16*2 + 20*2 + 20*16, BabyBear
# 8*16*4 + 13*4 + 13*16.  One Montgomery product ~ 4 IMAD-pipe instructions.
PERM_MODMULS = {0: 8 * 16 * 2 + 20 * 2 + 20 * 16, 1: 8 * 16 * 4 + 13 * 4 + 13 * 16}
IMAD_PER_MODMUL = 4
IMAD_PER_SM_CLK = 64
# DRAM bytes per algorithmic byte of one leaf-hashing launch (dram__bytes_read
# + dram__bytes_write over rows * (4 * width + 32)), from an ncu capture of
# k_hash_rows on a 2^23-row x 16-column LDE (the single-kb-2^22x16 workload)
HASH_TRAFFIC_RATIO = 0.966
# DRAM bytes per algorithmic byte (input + output) of one three-pass LDE, from
# an ncu capture of k_lde_a/b/c on a 2^22 x 16 matrix at split 2^11 x 2^11:
# 2,305 MB (read + write over the three passes) for 805 MB algorithmic.  The
# intermediate matrices T1 (n x w) and T2 (N x w) are each written once and
# read once.  One-pass matrices (n <= 2^11) move about their algorithmic bytes.
LDE_TRAFFIC_RATIO = 2305 / 805


GOLDEN_ROOTS = ROOT / "tests" / "golden" / "config_roots.json"
DEFAULT_WORKLOAD = "uneven-kb-2^30"


def root_parity(workload: str, seed: int, roots: dict) -> dict:
    """The roots the timed steps committed to (device inputs, plain form, host
    inputs), compared after timing with the root the CPU oracle computed for
    the same seeded inputs (tests/golden/config_roots.json)."""
    gold = json.loads(GOLDEN_ROOTS.read_text()).get(workload) if GOLDEN_ROOTS.exists() else None
    if gold is None or gold["seeds"][0] != seed * 1000:
        return {"checked": False, "why": "no oracle root for this workload and seed"}
    ok = {tag: r == gold["root"] for tag, r in roots.items()}
    return {"checked": True, "root_matches_oracle": all(ok.values()), "per_form": ok,
            "golden": "tests/golden/config_roots.json (CPU oracle, same seeded inputs)"}


def dist_setup(n_gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def allmax(world, v: float) -> float:
    """Max of v over the ranks (the slowest replica sets the job's time)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Each replica commits its own shard: a distinct seed per rank."""
    return base + 7919 * rank


def job_rate(world: int, cells_per_rank: int, steps: int, max_ms: float) -> float:
    """Whole-job throughput: the cells every rank committed over the slowest rank's time."""
    return world * cells_per_rank * steps / (max_ms / 1e3)


# ---------------------------------------------------------------- CPU legs
# The CPU legs commit a fixed, bounded sample of the workload: its smallest
# matrices first, up to CPU_SAMPLE_CELLS trace cells (about 10 s on 16 host
# threads for the uneven KoalaBear shard).  The GPU leg also times a commit of
# exactly these matrices, so the two rates compare the same work.
CPU_SAMPLE_CELLS = 1 << 26


def cpu_sample(shapes, max_cells: int = CPU_SAMPLE_CELLS):
    """Indices of the sampled matrices (the workload's own order) and their cells."""
    chosen, tot = [], 0
    for i in sorted(range(len(shapes)), key=lambda i: (shapes[i][1] << shapes[i][0], i)):
        c = shapes[i][1] << shapes[i][0]
        if tot + c > max_cells and chosen:
            break
        chosen.append(i)
        tot += c
    return sorted(chosen), tot


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_cpu(shapes, field, log_blowup, seed, steps, warmup, max_cells=CPU_SAMPLE_CELLS):
    """The oracle's TwoAdicFriPcs::commit on the CPU sample (same seeded
    matrices as the GPU commits), all host threads; median over `steps` runs."""
    from oracle import cpu as orc
    from pico_b200 import fields as F

    idx, cells = cpu_sample(shapes, max_cells)
    mats = [orc.random_matrix(field, shapes[i][0], shapes[i][1], seed * 1000 + i) for i in idx]
    shifts = [F.lde_shift(field)] * len(mats)
    for _ in range(warmup):
        orc.pcs_commit(field, mats, shifts, log_blowup)
    times = []
    for _ in range(max(steps, 1)):
        t = time.perf_counter()
        orc.pcs_commit(field, mats, shifts, log_blowup)
        times.append(time.perf_counter() - t)
    med = float(np.median(times))
    return {
        "value": cells / med,
        "unit": UNIT,
        "cores": orc.num_threads(),
        "cpu_model": cpu_model(),
        "sample": f"{len(idx)} of {len(shapes)} matrices of the workload (smallest first, at most "
                  f"{max_cells} cells): {cells} trace cells, the workload's own seeded inputs; "
                  f"median of {len(times)} runs",
        "seconds_per_run": med,
    }


# ---------------------------------------------------------------- GPU leg
def run_gpu(args, rank, world, local):
    import torch

    from pico_b200 import GpuContext, TwoAdicDomain, TwoAdicFriPcs
    from pico_b200 import fields as F
    from pico_b200.pcs import last_commit_stats

    wl = WORKLOADS[args.workload]
    field, b = wl["field"], wl["log_blowup"]
    shapes = wl["shapes"]()
    seed = replica_seed(wl["seed"], rank)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    traces = [F.random_matrix_torch(field, lh, w, seed * 1000 + i, dev) for i, (lh, w) in enumerate(shapes)]
    torch.cuda.synchronize()
    cells = sum(w << lh for lh, w in shapes)
    in_bytes = 4 * cells

    ctx = GpuContext(local)
    # autotune the LDE splits over the workload's heights and the hashing block size
    heights = [lh for lh, _ in shapes]
    tuned = ctx.autotune(field, max(12, min(heights)), max(12, max(heights))) if not args.no_tune else None
    pcs = TwoAdicFriPcs(ctx, field, b)
    doms = [TwoAdicDomain(lh) for lh, _ in shapes]

    def step(inputs, plain=False):
        root, _ = pcs.commit(list(zip(doms, inputs)), plain=plain, keep=False)
        return root, last_commit_stats()

    roots = {}

    def timed(inputs, plain=False, tag="device"):
        for _ in range(args.warmup):
            step(inputs, plain)
        barrier(world)
        torch.cuda.synchronize()
        sampler = ClockSampler(local)
        sampler.start()
        sampler.wait_first()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        stats = []
        for _ in range(args.steps):
            root, st = step(inputs, plain)
            stats.append(st)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        clocks = sampler.stop()
        barrier(world)
        ms = allmax(world, e0.elapsed_time(e1))
        roots[tag] = root.tolist()  # the last timed step's root, checked after timing
        return ms, stats, clocks

    ms, stats, clocks = timed(traces)
    ms_step = ms / args.steps
    value = job_rate(world, cells, args.steps, ms)

    # plain per-matrix form (the baseline form), same inputs
    ms_plain, _, _ = timed(traces, plain=True, tag="plain") if not args.skip_plain else (None, None, None)

    # the CPU legs' sample, committed on the GPU: the same matrices, so the
    # GPU/CPU ratio compares equal work
    idx, sample_cells = cpu_sample(shapes, args.cpu_cells)
    sample_in = [traces[i] for i in idx]
    sample_pcs_doms = [doms[i] for i in idx]

    def sample_step():
        pcs.commit(list(zip(sample_pcs_doms, sample_in)), keep=False)

    for _ in range(args.warmup):
        sample_step()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    for _ in range(args.steps):
        sample_step()
    s1.record()
    s1.synchronize()
    sample_ms = s0.elapsed_time(s1) / args.steps
    del sample_in

    # LDE kernels alone (no hashing sharing the SMs): every matrix of the
    # workload through coset_lde_batch, device in and out
    lde_only_ms = None
    if not args.skip_lde:
        from pico_b200 import Radix2DitParallel

        dft = Radix2DitParallel(ctx, field)
        shift = F.lde_shift(field)
        outs = [torch.empty((1 << (lh + b), w), dtype=torch.int32, device=dev) for lh, w in shapes]

        def lde_all():
            for t, o in zip(traces, outs):
                if t.numel():
                    dft.coset_lde_batch_bitrev(t, b, shift, out=o)

        lde_all()
        torch.cuda.synchronize()
        l0, l1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0.record()
        for _ in range(args.steps):
            lde_all()
        l1.record()
        l1.synchronize()
        lde_only_ms = l0.elapsed_time(l1) / args.steps
        del outs
        torch.cuda.empty_cache()

    # e2e: pinned host inputs through the C ABI, copies inside the timed region
    e2e = None
    if not args.skip_e2e:
        host = [t.cpu().pin_memory().numpy().view(np.uint32) for t in traces]
        del traces
        torch.cuda.empty_cache()
        ms_e2e, st_e2e, _ = timed(host, tag="host")
        e2e = {
            "value": world * cells * args.steps / (ms_e2e / 1e3),
            "unit": UNIT,
            "h2d_bytes_per_step": in_bytes,
            "d2h_bytes_per_step": 32,
            "ms_per_step": ms_e2e / args.steps,
            "h2d_ms_per_step": float(np.mean([s["h2d_ms"] for s in st_e2e])),
        }

    # roofline of the dominant kernel: Poseidon2 leaf hashing (integer-multiply bound)
    s0 = stats[-1]
    leaves_s = float(np.mean([s["leaves_ms"] for s in stats])) / 1e3
    mhz = clocks["sm_mhz"] or 1965.0
    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count
    imad_peak = sm_count * IMAD_PER_SM_CLK * mhz * 1e6 / 1e12  # Tops/s
    imad_ach = s0["leaf_permutations"] * PERM_MODMULS[field] * IMAD_PER_MODMUL / leaves_s / 1e12
    leaf_rows = 1 << max(lh for lh, _ in shapes) + b
    leaf_width = sum(w for lh, w in shapes if lh == max(l for l, _ in shapes))
    leaf_bytes = leaf_rows * (4 * leaf_width + 32)
    hbm_peak, hbm_kind = peaks()
    lde_alg_bytes = 4 * sum(w * ((1 << lh) + (1 << (lh + b))) for lh, w in shapes)
    lde_ach = lde_alg_bytes / (lde_only_ms / 1e3) / 1e9 if lde_only_ms else None
    lde_modmuls = sum(w * (((1 << lh) // 2) * lh * (1 + (1 << b)) + ((1 << lh) << b)) for lh, w in shapes)
    lde_imad = lde_modmuls * IMAD_PER_MODMUL / (lde_only_ms / 1e3) / 1e12 if lde_only_ms else None
    result = {
        "metric": METRIC,
        "value": value,
        "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32 (Montgomery-form KoalaBear field elements)" if field == 0 else "u32 (BabyBear)",
        "data": "synthetic: seeded uniform field elements (SplitMix64), no public dataset for this path",
        "config": {
            "workload": args.workload,
            "matrices": len(shapes),
            "trace_cells": cells,
            "log_blowup": b,
            "field": F.NAMES[field],
            "form": "batched",
            "parallelism": f"replicas x{world}",
            "l2": f"inputs ({in_bytes / 2**30:.2f} GiB) larger than L2 (126 MB); no flush"
                  if in_bytes > 126e6 else "inputs smaller than L2: not flushed",
            "autotuned": None if tuned is None else {
                "lde_log_n1": {str(k): v["log_n1"] for k, v in tuned.items() if k != "hash_block"},
                "hash_block": min(tuned["hash_block"], key=tuned["hash_block"].get)},
        },
        "gpu_launches": int(sum(s["launches"] for s in stats)),
        "clocks": clocks,
        "roofline": {
            "kernel": "k_hash_rows (Poseidon2 leaf hashing, one launch per commit)",
            "bound": "imad",
            "achieved": imad_ach,
            "peak": imad_peak,
            "unit": "Tops/s",
            "frac": imad_ach / imad_peak,
            "traffic": leaf_bytes * HASH_TRAFFIC_RATIO,
            "algorithmic_bytes": leaf_bytes,
            "launch_ms": leaves_s * 1e3,
            "note": f"integer-multiply bound: achieved = {IMAD_PER_MODMUL} IMAD x {PERM_MODMULS[field]} modmuls "
                    f"x leaf permutations / launch time; peak = {sm_count} SMs x {IMAD_PER_SM_CLK} IMAD/clk x "
                    f"median SM clock; traffic = algorithmic bytes x the DRAM/algorithmic ratio ncu measured",
        },
        "roofline_lde": {
            "kernel": "LDE kernels (k_pow_tables + k_lde_*), timed alone through coset_lde_batch",
            "bound": "hbm",
            "achieved": lde_ach,
            "peak": hbm_peak,
            "unit": "GB/s",
            "frac": lde_ach / hbm_peak if lde_ach else None,
            "traffic": lde_alg_bytes * LDE_TRAFFIC_RATIO if lde_alg_bytes else None,
            "traffic_note": "algorithmic bytes x the three-pass DRAM/algorithmic ratio ncu measured on a "
                            "2^22 x 16 LDE (T1 and T2 written and read once each); upper bound for "
                            "batches that hold one-pass matrices",
            "algorithmic_bytes": lde_alg_bytes,
            "ms": lde_only_ms,
            "peak_source": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback",
        },
        # the same LDE time against the integer-multiply peak: algorithmic Montgomery
        # products per column = twiddle products of the inverse and 2^b forward
        # transforms, (n/2) log2 n each, plus the n 2^b coset scalings
        "roofline_lde_imad": None if not lde_only_ms else {
            "kernel": "LDE kernels, timed alone (as roofline_lde)",
            "bound": "imad",
            "achieved": lde_imad,
            "peak": imad_peak,
            "unit": "Tops/s",
            "frac": lde_imad / imad_peak,
            "modmuls": lde_modmuls,
            "note": f"achieved = {IMAD_PER_MODMUL} IMAD x algorithmic Montgomery products / LDE time; the kernels "
                    f"also spend issue slots on modular additions, shared-memory traffic and index arithmetic",
        },
        "phases_ms": {k: float(np.mean([s[k] for s in stats])) for k in ("lde_ms", "leaves_ms", "tree_ms", "total_ms")},
        "e2e": e2e,
        "parity": root_parity(args.workload, seed, roots),
        "on_cpu_sample": {"value": sample_cells / (sample_ms / 1e3), "unit": UNIT, "ms_per_step": sample_ms,
                          "matrices": len(idx), "trace_cells": sample_cells,
                          "what": "the same commit on the cpu_baseline's sample of matrices (device inputs)"},
    }
    if ms_plain is not None:
        result["plain_form"] = {"value": world * cells * args.steps / (ms_plain / 1e3),
                                "ms_per_step": ms_plain / args.steps}
    if args.workload == DEFAULT_WORKLOAD and world == 1 and not args.skip_c1:
        result["c1"] = c1_summary(ctx, args, local)
    ctx.close()
    return result, shapes, field, b


C1_WORKLOAD = "single-kb-2^16x64"
C1_STEPS = 50


def c1_summary(ctx, args, local):
    """The single-matrix KoalaBear commit (2^16 x 64, blowup 2): device-resident
    and end-to-end rates over C1_STEPS commits each (five timed groups, the
    median group's time per commit), the CPU oracle on the same whole commit
    (all host threads, median of 5), the ratios, and the root against the
    oracle's golden."""
    import torch

    from pico_b200 import TwoAdicDomain, TwoAdicFriPcs
    from pico_b200 import fields as F
    from pico_b200.pcs import last_commit_stats

    wl = WORKLOADS[C1_WORKLOAD]
    field, b, shapes, seed = wl["field"], wl["log_blowup"], wl["shapes"](), wl["seed"]
    dev = torch.device("cuda", local)
    traces = [F.random_matrix_torch(field, lh, w, seed * 1000 + i, dev) for i, (lh, w) in enumerate(shapes)]
    host = [t.cpu().pin_memory().numpy().view(np.uint32) for t in traces]
    cells = sum(w << lh for lh, w in shapes)
    pcs = TwoAdicFriPcs(ctx, field, b)
    doms = [TwoAdicDomain(lh) for lh, _ in shapes]
    out = {}
    for tag, inputs in (("device", traces), ("host", host)):
        for _ in range(max(args.warmup, 3)):
            pcs.commit(list(zip(doms, inputs)), keep=False)
        torch.cuda.synchronize()
        groups = []  # C1_STEPS commits in five timed groups; the median group's rate
        for _ in range(5):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(C1_STEPS // 5):
                root, _ = pcs.commit(list(zip(doms, inputs)), keep=False)
            e1.record()
            e1.synchronize()
            groups.append(e0.elapsed_time(e1) / (C1_STEPS // 5))
        out[tag] = (float(np.median(groups)), root.tolist(), [round(g, 4) for g in groups])
        if tag == "host":
            last = last_commit_stats()  # the last commit's own device timeline
            host_phases = {"h2d_ms": last["h2d_ms"], "device_total_ms": last["total_ms"]}
    cpu = run_cpu(shapes, field, b, seed, 5, 1, max_cells=cells)
    ms_dev, ms_e2e = out["device"][0], out["host"][0]
    return {
        "workload": C1_WORKLOAD, "trace_cells": cells, "log_blowup": b, "steps": C1_STEPS,
        "value": cells / (ms_dev / 1e3), "ms_per_step": ms_dev,
        "e2e": {"value": cells / (ms_e2e / 1e3), "unit": UNIT, "ms_per_step": ms_e2e,
                "h2d_bytes_per_step": 4 * cells, "d2h_bytes_per_step": 32, **host_phases},
        "cpu_baseline": cpu,
        "gpu_over_cpu": cells / (ms_dev / 1e3) / cpu["value"],
        "gpu_over_cpu_e2e": cells / (ms_e2e / 1e3) / cpu["value"],
        "ms_per_step_groups": {tag: g for tag, (_, _, g) in out.items()},
        "parity": root_parity(C1_WORKLOAD, seed, {tag: r for tag, (_, r, _) in out.items()}),
        "l2": "input 16 MiB, LDE 32 MiB: smaller than L2, not flushed (the size the config names)",
    }


# ---------------------------------------------------------------- opening leg
OPEN_METRIC = ("opened trace cells/sec (TwoAdicFriPcs::open: opened values, reduced openings, FRI commit "
               "phase, proof of work, query records; bit-exact)")


def open_points(field, shapes, seed: int = 6):
    """Pico's main-trace opening points: zeta and zeta * w_n for each trace of height n."""
    from pico_b200 import fields as F

    p = F.P[field]
    rng = np.random.default_rng(seed)
    zc = [int(v) for v in rng.integers(0, p, size=4)]
    zeta = np.array([F.monty(field, v) for v in zc], dtype=np.uint32)
    pts = []
    for lh, _ in shapes:
        w = F.two_adic_generator(field, lh)
        nxt = np.array([F.monty(field, v * w % p) for v in zc], dtype=np.uint32)
        pts.append(np.stack([zeta, nxt]))
    return pts


def run_cpu_open(shapes, field, b, seed, steps, warmup, seconds, nq=84, pow_bits=16):
    """The oracle's TwoAdicFriPcs::open on a bounded sample (smallest matrices
    first, sized by a probe to about `seconds` per run); the commit it opens is
    made outside the timed region."""
    from oracle import cpu as orc
    from pico_b200 import fields as F

    probe_shape = [(12, 16)]
    pm = [F.random_matrix(field, 12, 16, 5)]
    root, ldes, layers = orc.pcs_commit(field, pm, [F.lde_shift(field)], b, want_ldes=True, want_layers=True)
    pb = [{"ldes": ldes, "points": open_points(field, probe_shape), "layers": layers}]
    t = time.perf_counter()
    orc.pcs_open(field, pb, b, nq, pow_bits)
    fixed = time.perf_counter() - t  # proof of work and queries dominate a tiny open
    t = time.perf_counter()
    orc.pcs_open(field, pb, b, nq, 0)
    rate = (16 << 12) / max(time.perf_counter() - t, 1e-6)
    budget = rate * max(seconds - fixed, 1.0)
    chosen, tot = [], 0
    for lh, w in sorted(shapes, key=lambda s: s[1] << s[0]):
        if tot + (w << lh) > budget and chosen:
            break
        chosen.append((lh, w))
        tot += w << lh
    mats = [F.random_matrix(field, lh, w, seed * 1000 + i) for i, (lh, w) in enumerate(chosen)]
    root, ldes, layers = orc.pcs_commit(field, mats, [F.lde_shift(field)] * len(mats), b, want_ldes=True,
                                        want_layers=True)
    batch = [{"ldes": ldes, "points": open_points(field, chosen), "layers": layers}]
    for _ in range(warmup):
        orc.pcs_open(field, batch, b, nq, pow_bits)
    times = []
    for _ in range(steps):
        t = time.perf_counter()
        orc.pcs_open(field, batch, b, nq, pow_bits)
        times.append(time.perf_counter() - t)
    med = float(np.median(times))
    return {"value": tot / med, "unit": UNIT, "cores": orc.num_threads(),
            "sample": f"open of {len(chosen)} of {len(shapes)} matrices of the workload (smallest first), "
                      f"{tot} trace cells, 2 points each, {nq} queries, {pow_bits} proof-of-work bits; "
                      f"median of {steps} runs",
            "seconds_per_run": med}


OPEN_WORKLOADS = {
    "open-kb-2^30": lambda: uneven_kb_shapes(),
    # the same distribution at 2^25 cells (heights 2^6..2^18): for profiler captures
    "open-kb-2^25": lambda: uneven_kb_shapes(target_log=25, lo=6, hi=18),
}


def run_open(args, rank, world, local):
    """Open the uneven KoalaBear shard's commitment (2^30 trace cells, 32
    traces) at Pico's main-trace points: every trace at zeta and zeta * w_n;
    84 queries, 16 proof-of-work bits, log_blowup 1 (KoalaBearPoseidon2's FRI
    configuration, vm/src/configs/stark_config/kb_poseidon2.rs:62-72).  One
    step = one pcs.open on the resident commitment."""
    import torch

    from pico_b200 import GpuContext, TwoAdicDomain, TwoAdicFriPcs, abi
    from pico_b200 import fields as F

    field, b, nq, pow_bits = 0, 1, 84, 16
    shapes = OPEN_WORKLOADS[args.workload]()
    seed = replica_seed(2, rank)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    traces = [F.random_matrix_torch(field, lh, w, seed * 1000 + i, dev) for i, (lh, w) in enumerate(shapes)]
    torch.cuda.synchronize()
    cells = sum(w << lh for lh, w in shapes)
    ctx = GpuContext(local)
    if not args.no_tune:
        heights = [lh for lh, _ in shapes]
        ctx.autotune(field, max(12, min(heights)), max(12, max(heights)))
    pcs = TwoAdicFriPcs(ctx, field, b)
    doms = [TwoAdicDomain(lh) for lh, _ in shapes]
    root, pd = pcs.commit(list(zip(doms, traces)))
    pts = open_points(field, shapes)
    rounds = [(pd, pts)]

    def step():
        return pcs.open(rounds, abi.Challenger(), num_queries=nq, proof_of_work_bits=pow_bits)

    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    sampler.wait_first()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    outs = [step() for _ in range(args.steps)]
    e1.record()
    e1.synchronize()
    clocks = sampler.stop()
    barrier(world)
    ms = allmax(world, e0.elapsed_time(e1))
    st = outs[-1]["stats"]
    proof_bytes = 4 * (outs[-1]["values"].size + outs[-1]["roots"].size + outs[-1]["queries"].size + 4 + 1 + nq)

    # roofline of the reduction phase: the low-coset cells read once, the
    # inverse denominators of both points read per low-coset row, and the
    # reduced opening (extended from the low coset) written per committed row
    heights = sorted({lh + b for lh, _ in shapes})
    red_bytes = 4 * st["reduce_cells"] + sum((1 << (h - b)) * 16 * 2 + (1 << h) * 16 for h in heights)
    hbm_peak, hbm_kind = peaks()
    red_ach = red_bytes / (st["ms_reduce"] / 1e3) / 1e9
    val_bytes = 4 * st["value_cells"] // 2 + sum(16 * (1 << lh) * 2 for lh, _ in shapes)

    # e2e: commit from pinned host traces and open, per step
    e2e = None
    if not args.skip_e2e:
        host = [t.cpu().pin_memory().numpy().view(np.uint32) for t in traces]
        pd.release()
        del traces
        torch.cuda.empty_cache()

        def e2e_step():
            _, pdh = pcs.commit(list(zip(doms, host)))
            out = pcs.open([(pdh, pts)], abi.Challenger(), num_queries=nq, proof_of_work_bits=pow_bits)
            pdh.release()
            return out

        for _ in range(max(1, args.warmup - 1)):
            e2e_step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        ms_e2e = allmax(world, (time.perf_counter() - t0) * 1e3)
        e2e = {"value": world * cells * args.steps / (ms_e2e / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": 4 * cells, "d2h_bytes_per_step": proof_bytes + 32,
               "ms_per_step": ms_e2e / args.steps,
               "what": "commit from pinned host traces + open, both through the C ABI (host wall clock)"}
    ctx.close()
    return {
        "metric": OPEN_METRIC, "value": job_rate(world, cells, args.steps, ms), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32 (Montgomery-form KoalaBear, EF4 challenges)",
        "data": "synthetic: seeded uniform field elements; random zeta",
        "config": {"workload": args.workload, "matrices": len(shapes), "trace_cells": cells, "log_blowup": b,
                   "points_per_matrix": 2, "num_queries": nq, "proof_of_work_bits": pow_bits,
                   "l2": f"committed LDEs ({8 * cells / 2**30:.2f} GiB) larger than L2 (126 MB); no flush"},
        "gpu_launches": int(st["launches"]) * args.steps,
        "clocks": clocks,
        "phases_ms": {k: st[k] for k in ("ms_values", "ms_reduce", "ms_fri", "ms_grind", "ms_queries", "ms_total")},
        "roofline": {
            "kernel": "reduction phase: k_reduce and k_reduce_combine over the low coset, LDE of the result",
            "bound": "hbm",
            "achieved": red_ach, "peak": hbm_peak, "unit": "GB/s", "frac": red_ach / hbm_peak, "traffic": None,
            "algorithmic_bytes": red_bytes, "launch_ms": st["ms_reduce"],
            "peak_source": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback"},
        "roofline_values": {
            "kernel": "k_inv_denoms + k_open_partial + k_open_finalize (opened values)", "bound": "hbm",
            "achieved": val_bytes / (st["ms_values"] / 1e3) / 1e9, "peak": hbm_peak, "unit": "GB/s",
            "frac": val_bytes / (st["ms_values"] / 1e3) / 1e9 / hbm_peak, "algorithmic_bytes": val_bytes,
            "launch_ms": st["ms_values"]},
        "e2e": e2e,
    }


# ---------------------------------------------------------------- FRI leg
def fri_launches(log_n: int, rounds: int, log_final_len: int) -> int:
    """Kernels one commit phase launches (the round loop of fri_host.cu): the
    first round's leaf hashing; per round the wide compression levels one
    launch each, seven narrow levels per subtree launch, the tree top with the
    challenger step, and the fold (with the next leaves); then the final
    observation (and the final polynomial when it keeps coefficients)."""
    nl = 0
    for r in range(rounds):
        n = 1 << (log_n - r - 1)
        nl += 1 if r == 0 else 0
        while n > 512:
            nl += 1
            n = n >> 7 if n <= (1 << 15) else n // 2
        nl += 2
    return nl + (1 if log_final_len == 0 else 2)


def run_fri(args):
    """FRI commit phase on a device-resident KoalaBear EF4 codeword of 2^23
    evaluations (a degree < 2^22 random polynomial, coset LDE with blowup 2):
    per round Poseidon2 Merkle commit of the (len/2) x 2 extension matrix,
    on-device challenger, arity-2 fold; all layers stay resident.  Two
    stopping rules: the reference's (fold to 2^log_blowup, single final
    element) and 2^4 final coefficients."""
    import torch

    from pico_b200 import GpuContext, Radix2DitParallel, TwoAdicFriPcs
    from pico_b200 import fields as F

    f, log_trace, b = 0, 22, 1
    dev = torch.device("cuda", 0)
    ctx = GpuContext(0)
    base = F.random_matrix_torch(f, log_trace, 4, 4000, dev)
    cw = torch.empty((1 << (log_trace + b), 4), dtype=torch.int32, device=dev)
    Radix2DitParallel(ctx, f).coset_lde_batch_bitrev(base, b, F.lde_shift(f), out=cw)
    torch.cuda.synchronize()
    pcs = TwoAdicFriPcs(ctx, f, b)
    out = {}
    clocks = None
    for name, lf in (("final_1", 0), ("final_16", 4)):
        for _ in range(args.warmup):
            pcs.fri_commit_phase(cw, log_final_len=lf)
        torch.cuda.synchronize()
        if name == "final_1":
            sampler = ClockSampler(0)
            sampler.start()
            sampler.wait_first()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            res = pcs.fri_commit_phase(cw, log_final_len=lf)
        torch.cuda.synchronize()
        e1.record()
        e1.synchronize()
        if name == "final_1":
            clocks = sampler.stop()
        ms = e0.elapsed_time(e1) / args.steps
        out[name] = {"ms": ms, "rounds": res.rounds, "elements_per_s": (1 << (log_trace + b)) / (ms / 1e3)}
        gold = json.loads(GOLDEN_ROOTS.read_text()).get("fri-kb-2^23") if GOLDEN_ROOTS.exists() else None
        if gold is not None:  # the last timed step's roots, betas and final values against the oracle's
            g = gold[name]
            out[name]["matches_oracle"] = (res.roots.tolist() == g["roots"] and res.betas.tolist() == g["betas"]
                                           and res.final_poly.tolist() == g["final"])
    # end to end: the codeword from pinned host memory, roots, betas and the
    # final polynomial back to the host, per call
    n_el = 1 << (log_trace + b)
    cw_host = torch.empty((n_el, 4), dtype=torch.int32, pin_memory=True)
    cw_host.copy_(cw)
    cw_np = cw_host.numpy().view(np.uint32)
    for _ in range(args.warmup):
        pcs.fri_commit_phase(cw_np)
    t = time.perf_counter()
    for _ in range(args.steps):
        pcs.fri_commit_phase(cw_np)
    e2e_s = (time.perf_counter() - t) / args.steps
    rounds = out["final_1"]["rounds"]
    ctx.close()
    # Poseidon2 work of a phase: per round, one permutation per leaf (two EF4
    # elements = eight words) and one per internal node of the round's tree
    perms = sum((1 << (log_trace + b - 1 - r)) + (1 << (log_trace + b - 1 - r)) - 1 for r in range(rounds))
    imad_peak = 148 * IMAD_PER_SM_CLK * ((clocks or {}).get("sm_mhz") or 1965.0) / 1e6
    imad_ach = perms * PERM_MODMULS[f] * IMAD_PER_MODMUL / (out["final_1"]["ms"] / 1e3) / 1e12
    # CPU: the oracle's commit phase of a 2^17-element codeword of the same kind
    from oracle import cpu as orc

    small = 19
    cw_small = orc.coset_lde(f, orc.random_matrix(f, small, 4, 4001), b, F.lde_shift(f))
    runs = []
    for _ in range(3):
        t = time.perf_counter()
        orc.fri_commit_phase(f, cw_small, b, 0)
        runs.append(time.perf_counter() - t)
    cpu_s = float(np.median(runs))
    return {
        "metric": "FRI commit-phase codeword elements/sec (EF4, arity 2, Poseidon2 layer commits)",
        "value": out["final_1"]["elements_per_s"], "unit": "elements/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": out["final_1"]["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 (KoalaBear EF4)", "data": "synthetic: random degree < 2^22 EF4 polynomial",
        "config": {"workload": "fri-kb-2^23", "log_n": log_trace + b, "log_blowup": b,
                   "l2": "codeword 128 MiB and its layers exceed L2 (126 MB); no flush"},
        "modes": out,
        "clocks": clocks,
        "gpu_launches": args.steps * fri_launches(log_trace + b, rounds, 0),
        "e2e": {"value": n_el / e2e_s, "unit": "elements/s", "ms_per_step": e2e_s * 1e3,
                "h2d_bytes_per_step": n_el * 16, "d2h_bytes_per_step": rounds * 48 + 16},
        "roofline": {"kernel": "the phase's Poseidon2 kernels (k_fri_fold_hash, k_compress, k_subtree_quad, "
                               "k_tree_top)", "bound": "imad", "achieved": imad_ach, "peak": imad_peak,
                     "unit": "Tops/s", "frac": imad_ach / imad_peak, "traffic": None, "permutations": perms,
                     "note": "survey model: 4 IMAD x modmuls per permutation; the phase is bound by chains of "
                             "dependent permutations (each round's leaves need the previous round's beta)"},
        "cpu_baseline": {"value": (1 << (small + b)) / cpu_s, "unit": "elements/s", "cores": orc.num_threads(),
                         "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"the oracle's commit phase of a 2^{small + b}-element codeword, median of 3"},
    }


# ---------------------------------------------------------------- quotient leg
def chip_program(field, main_w: int = 32, seed: int = 9):
    """A synthetic chip's constraints shaped like Pico's (no public dataset):
    16 degree-2 products wired across the main columns, 8 transition
    constraints, 4 boolean checks, first-row and last-row constraints, and a
    LogUp-style running sum in one permutation column:
    (z' - z) (ch0 + x0 + ch1 x1) = x2 on transitions, z = regional sum on the
    first row."""
    from pico_b200.quotient import ConstraintBuilder

    rng = np.random.default_rng(seed)
    b = ConstraintBuilder()
    m = lambda c, nxt=False: b.main(int(c), nxt)
    for i in range(16):
        a, c, d = rng.integers(0, main_w, size=3)
        b.assert_zero(m(a) * m(c) - m(d))
    for i in range(8):
        a, c = rng.integers(0, main_w, size=2)
        b.when_transition().assert_eq(m(i, True), m(a) + m(c))
    for i in range(4):
        x = m(24 + i)
        b.assert_zero(x * (x - 1))
    b.when_first_row().assert_eq(m(0), b.public(0))
    b.when_last_row().assert_eq(m(1), b.public(1))
    z, zn = b.permutation(0), b.permutation(0, True)
    b.when_transition().assert_zero((zn - z) * (b.challenge(0) + m(0) + b.challenge(1) * m(1)) - m(2))
    b.when_first_row().assert_zero(z - b.regional_cumulative_sum())
    return b.program(field)


def run_quotient(args):
    """compute_quotient_values of the synthetic chip over one 2^20-row
    KoalaBear trace of 32 columns plus one extension permutation column,
    quotient degree 2 (2^21 points), the traces resident from their commits.
    One step = one pico_gpu_quotient_values call with device output."""
    import torch

    from pico_b200 import GpuContext, TwoAdicDomain, TwoAdicFriPcs
    from pico_b200 import fields as F
    from pico_b200.quotient import compute_quotient_values
    from oracle import cpu as orc

    f, logn, log_qd, main_w = 0, 20, 1, 32
    prog = chip_program(f, main_w)
    dev = torch.device("cuda", 0)
    ctx = GpuContext(0)
    pcs = TwoAdicFriPcs(ctx, f, 1)
    main = F.random_matrix_torch(f, logn, main_w, 9100, dev)
    perm = F.random_matrix_torch(f, logn, 4, 9101, dev).reshape(1 << logn, 1, 4)
    _, pd = pcs.commit([(TwoAdicDomain(logn), main), (TwoAdicDomain(logn), perm)])
    pub = F.to_monty(f, [1, 2])
    chal = F.to_monty(f, F.uniform(f, 8, 9102)).reshape(2, 4)
    reg = F.to_monty(f, F.uniform(f, 4, 9103))
    alpha = F.to_monty(f, F.uniform(f, 4, 9104))
    Q = 1 << (logn + log_qd)
    out = torch.empty((Q, 4), dtype=torch.int32, device=dev)

    def step():
        compute_quotient_values(ctx, prog, logn, log_qd, (pd, 0), permutation=(pd, 1), public_values=pub,
                                perm_challenges=chal, regional_sum=reg, alpha=alpha, out=out)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(0)
    sampler.start()
    sampler.wait_first()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    e1.synchronize()
    clocks = sampler.stop()
    ms = e0.elapsed_time(e1) / args.steps
    # parity of the timed output on a slice of points, against the oracle (its
    # own LDE of the same traces, natural order)
    got = out.cpu().numpy().view(np.uint32)
    main_h = main.cpu().numpy().view(np.uint32)
    perm_h = perm.cpu().numpy().view(np.uint32)
    want = orc.quotient_values(f, logn, log_qd, prog, orc.on_quotient_domain(f, main_h, log_qd),
                               perm_q=orc.on_quotient_domain(f, perm_h, log_qd), public_values=pub,
                               perm_challenges=chal, regional_sum=reg, alpha=alpha)
    match = bool((got == want).all())
    # CPU: the oracle on a 2^14-row trace of the same program (per point)
    small = 14
    mh, ph = main_h[: 1 << small], perm_h[: 1 << small]
    mq, pq = orc.on_quotient_domain(f, mh, log_qd), orc.on_quotient_domain(f, ph, log_qd)
    t = time.perf_counter()
    orc.quotient_values(f, small, log_qd, prog, mq, perm_q=pq, public_values=pub, perm_challenges=chal,
                        regional_sum=reg, alpha=alpha)
    cpu_s = time.perf_counter() - t
    ctx.close()
    points = Q
    # algorithmic bytes: every point's main and permutation row read once (the
    # next-row reads are other points' rows) and its EF4 quotient written
    q_bytes = Q * 4 * (main_w + 4 + 4)
    hbm_peak, hbm_kind = peaks()
    q_ach = q_bytes / (ms / 1e3) / 1e9
    return {
        "metric": "quotient-domain points/sec (compute_quotient_values of one chip, resident LDEs)",
        "value": points / (ms / 1e3), "unit": "points/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 (KoalaBear, EF4 accumulator)", "data": "synthetic: seeded traces, a chip-shaped program",
        "config": {"workload": "quotient-kb-2^20", "log_trace": logn, "log_quotient_degree": log_qd,
                   "main_width": main_w, "perm_width": 1, "program_ops": int(prog.shape[0])},
        "parity": {"matches_oracle": match, "points": points},
        "clocks": clocks,
        "gpu_launches": args.steps,
        "roofline": {"kernel": "k_quotient", "bound": "hbm", "achieved": q_ach, "peak": hbm_peak, "unit": "GB/s",
                     "frac": q_ach / hbm_peak, "traffic": None, "algorithmic_bytes": q_bytes,
                     "peak_source": f"{hbm_kind} (MEASURED_PEAKS.json hbm_gbs)" if hbm_kind == "measured" else "fallback",
                     "note": "the kernel interprets the constraint program per point, so its instruction stream, not "
                             "HBM, bounds it; the fraction shows how far the trace reads are from limiting it"},
        "cpu_baseline": {"value": (2 << small) / cpu_s, "unit": "points/s", "cores": orc.num_threads(),
                         "kind": "port", "cpu_model": cpu_model(),
                         "sample": f"the same program on a 2^{small}-row trace ({2 << small} points), one run"},
    }


# ---------------------------------------------------------------- serving leg
# request mixes: (log2 heights low, high), widths (low, high)
SERVING_MIXES = {
    # traces of 2^12 .. 2^21 rows and 16 .. 512 columns
    "prover": ((12, 21), (16, 512)),
    # the same matrix counts with small traces (2^8 .. 2^13 rows, 8 .. 64 columns):
    # the regime where one launch per matrix costs more than the work
    "small": ((8, 13), (8, 64)),
}


def serving_requests(n_req: int, seed: int = 5, max_cells: int = 1 << 30, mix: str = "prover"):
    """Requests of 1..40 matrices, log2 heights uniform on [12, 21], widths
    uniform on [16, 512] (the "small" mix: heights 2^8..2^13, widths 8..64);
    70% KoalaBear / 30% BabyBear; log_blowup 1 or 2.  A request is cut to its
    first matrices totalling at most max_cells trace cells, so that one
    request (with its blowup-4 LDEs and scratch) fits HBM."""
    (hl, hh), (wl, wh) = SERVING_MIXES[mix]
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(n_req):
        k = int(rng.integers(1, 41))
        f = 0 if rng.random() < 0.7 else 1
        b = int(rng.integers(1, 3))
        shapes = [(int(rng.integers(hl, hh + 1)), int(rng.integers(wl, wh + 1))) for _ in range(k)]
        kept, tot = [], 0
        for lh, w in shapes:
            if kept and tot + (w << lh) > max_cells:
                break
            kept.append((lh, w))
            tot += w << lh
        reqs.append((f, b, kept))
    return reqs


def run_serving(args):
    """Poisson arrivals of commit requests into the serving queue (admission
    by free HBM, up to --slots requests on the device at once), for three
    forms: batched (each request alone on its stream), grouped (queued
    requests admitted together, up to --group of them sharing their LDE and
    row-hashing launches) and the plain one-matrix-per-launch form, at several
    offered loads (multiples of the plain form's one-at-a-time capacity, the
    same arrival times for every form); plus the batched and plain forms one
    at a time.  Inputs are views into a device-resident pool of seeded field
    elements.  The memory pool is grown before timing by one pass of every
    request (or the first --serve-warm), one at a time and served."""
    import threading as th

    import torch

    from pico_b200 import CommitServer, GpuContext, TwoAdicDomain, TwoAdicFriPcs
    from pico_b200 import fields as F

    dev = torch.device("cuda", 0)
    reqs = serving_requests(args.requests, mix=args.mix)
    pool_cells = 1 << 30
    pools = {f: F.random_matrix_torch(f, 30, 1, 5000 + f, dev).reshape(-1) for f in (0, 1)}

    def views(f, shapes, salt):
        rng = np.random.default_rng(salt)
        out = []
        for lh, w in shapes:
            cells = w << lh
            if cells > pool_cells:
                raise ValueError("matrix larger than the pool")
            off = int(rng.integers(0, (pool_cells - cells) // 4 + 1)) * 4
            out.append(pools[f][off:off + cells].view(1 << lh, w))
        return out

    mats = [views(f, shapes, 7 * i + 1) for i, (f, b, shapes) in enumerate(reqs)]
    cells = [sum(w << lh for lh, w in shapes) for (_, _, shapes) in reqs]
    total_cells = sum(cells)
    ctx = GpuContext(0, n_streams=8, max_inflight=args.slots, max_group=1)  # each request alone
    server = CommitServer(ctx)
    # the grouped form's context shares the device's memory pool and budget
    ctx_g = GpuContext(0, hbm_budget_bytes=ctx.memory()[1], n_streams=8, max_inflight=args.slots,
                       max_group=args.group)
    server_g = CommitServer(ctx_g)

    def sequential(plain):
        lat = []
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for (f, b, shapes), m in zip(reqs, mats):
            t = time.perf_counter()
            TwoAdicFriPcs(ctx, f, b).commit([(TwoAdicDomain(lh), x) for (lh, _), x in zip(shapes, m)], plain=plain,
                                            keep=False)
            lat.append(time.perf_counter() - t)
        return time.perf_counter() - t0, lat

    def served(plain, arrivals, server=server):
        handles = [None] * len(reqs)
        lat = [None] * len(reqs)
        queued = [None] * len(reqs)
        t0 = time.perf_counter()

        def waiter():
            for i in range(len(reqs)):
                while handles[i] is None:
                    time.sleep(0.0002)
                handles[i].wait(keep=False)
                q_us, run_us = handles[i].times()
                lat[i] = (q_us + run_us) / 1e6
                queued[i] = q_us / 1e6
                handles[i].free()

        wt = th.Thread(target=waiter)
        wt.start()
        for i, ((f, b, shapes), m) in enumerate(zip(reqs, mats)):
            now = time.perf_counter() - t0
            if arrivals[i] > now:
                time.sleep(arrivals[i] - now)
            handles[i] = server.submit(f, m, b, plain=plain)
        wt.join()
        return time.perf_counter() - t0, lat, queued

    def pct(x, q):
        return float(np.percentile(np.array(x) * 1e3, q))

    # grow the pool: every request once (or the first --serve-warm), one at a
    # time, then once served back to back
    # (all arriving at once, so the grouped form also reaches its largest
    # groups: a group holds its members' scratch at the same time, and the
    # pool grows, synchronously, the first time it needs more)
    def warm():
        sequential(False)
        served(False, np.zeros(len(reqs)))
        if args.group > 1:
            served(False, np.zeros(len(reqs)), server_g)

    if args.serve_warm == 0 or args.serve_warm >= len(reqs):
        warm()
    else:
        full = (reqs, mats)
        reqs, mats = reqs[:args.serve_warm], mats[:args.serve_warm]
        warm()
        reqs, mats = full
    seq_s, seq_lat = sequential(False)
    plain_s, plain_lat = sequential(True)
    cap_plain = total_cells / plain_s
    rng = np.random.default_rng(55)
    gaps = rng.exponential(1.0, size=len(reqs))  # unit-rate arrivals, scaled per load
    mean_cells = total_cells / len(reqs)
    sweep = []
    loads = [float(x) for x in args.loads.split(",")] if args.loads else [0.5, 1.0, 1.25]
    for load in sorted(set([args.load] + loads)):
        rate = load * cap_plain / mean_cells  # requests per second
        arrivals = np.cumsum(gaps / rate)
        row = {"offered_load_vs_plain_capacity": load, "poisson_rate_per_s": rate}
        forms = [("batched", False, server), ("plain", True, server)]
        if args.group > 1:
            forms.insert(1, ("grouped", False, server_g))
        for name, plain, srv in forms:
            s_, lat, queued = served(plain, arrivals, srv)
            row[name] = {"cells_per_s": total_cells / s_, "p50_ms": pct(lat, 50), "p90_ms": pct(lat, 90),
                         "p99_ms": pct(lat, 99), "max_ms": pct(lat, 100),
                         "mean_queue_ms": float(np.mean(queued) * 1e3)}
        sweep.append(row)
    ctx_g.close()
    ctx.close()
    main_row = next(r for r in sweep if r["offered_load_vs_plain_capacity"] == args.load)
    return {
        "metric": "served commit throughput (trace cells/sec) with p50/p99 latency",
        "value": main_row["batched"]["cells_per_s"], "unit": "cells/s", "n_gpus": 1, "steps": len(reqs),
        "warmup": 2 * len(reqs),
        "ms_per_step": total_cells / main_row["batched"]["cells_per_s"] * 1e3 / len(reqs),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic: views into a seeded device pool",
        "config": {"workload": "serving", "mix": args.mix, "requests": len(reqs), "slots": args.slots, "offered_load": args.load,
                   "max_group": args.group, "total_cells": total_cells},
        "served": main_row["batched"],
        "served_grouped": main_row.get("grouped"),
        "served_plain": main_row["plain"],
        "sweep": sweep,
        "one_at_a_time_batched": {"p50_ms": pct(seq_lat, 50), "p99_ms": pct(seq_lat, 99),
                                  "cells_per_s": total_cells / seq_s},
        "one_at_a_time_plain": {"p50_ms": pct(plain_lat, 50), "p99_ms": pct(plain_lat, 99),
                                "cells_per_s": cap_plain},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS) + ["fri-kb-2^23", "serving", "quotient-kb-2^20"]
                    + list(OPEN_WORKLOADS),
                    default=DEFAULT_WORKLOAD)
    ap.add_argument("--requests", type=int, default=60, help="serving: number of requests")
    ap.add_argument("--load", type=float, default=0.8,
                    help="serving: offered load vs the plain form's one-at-a-time capacity")
    ap.add_argument("--slots", type=int, default=2, help="serving: requests on the device at once")
    ap.add_argument("--group", type=int, default=8,
                    help="serving: largest group of queued requests sharing launches in the grouped form (1: none)")
    ap.add_argument("--mix", choices=list(SERVING_MIXES), default="prover", help="serving: request mix")
    ap.add_argument("--loads", default="", help="serving: extra offered loads to sweep, comma separated "
                                                  "(default 0.5,1.0,1.25)")
    ap.add_argument("--serve-warm", type=int, default=0,
                    help="serving: requests used to warm the memory pool (0: all of them)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="opening workloads: CPU sample size in seconds")
    ap.add_argument("--cpu-runs", type=int, default=5, help="runs of the CPU baseline (median)")
    ap.add_argument("--cpu-cells", type=int, default=CPU_SAMPLE_CELLS,
                    help="commit workloads: trace cells of the CPU sample (smallest matrices first)")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-plain", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-lde", action="store_true", help="skip the LDE-alone timing")
    ap.add_argument("--skip-c1", action="store_true", help="skip the single-matrix (2^16 x 64) summary key")
    ap.add_argument("--no-tune", action="store_true", help="default LDE splits and block size (no autotuning)")
    args = ap.parse_args()

    rank, world, local = dist_setup(args.gpus)
    if args.workload in OPEN_WORKLOADS:
        if args.impl == "reference":
            if rank == 0:
                ref = run_cpu_open(OPEN_WORKLOADS[args.workload](), 0, 1, 2, args.steps, args.warmup,
                                   args.cpu_seconds)
                print(json.dumps({
                    "metric": OPEN_METRIC, "value": ref["value"], "unit": UNIT, "impl": "reference",
                    "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                    "ms_per_step": ref["seconds_per_run"] * 1e3, "higher_is_better": True, "scaling": "weak",
                    "vs_baseline": None, "dtype": "u32", "data": "synthetic: seeded uniform field elements",
                    "config": {"workload": args.workload, "sample": ref["sample"]},
                    "cpu_baseline": {"value": ref["value"], "unit": UNIT, "cores": ref["cores"], "kind": "port",
                                     "sample": ref["sample"]},
                    "e2e": {"value": ref["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                }), flush=True)
            return
        res = run_open(args, rank, world, local)
        if rank == 0:
            if not args.skip_cpu:
                cpu = run_cpu_open(OPEN_WORKLOADS[args.workload](), 0, 1, 2, 1, 0, args.cpu_seconds)
                res["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                                       "sample": cpu["sample"]}
            print(json.dumps(res), flush=True)
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()
        return
    if args.workload in ("fri-kb-2^23", "serving", "quotient-kb-2^20"):
        if rank == 0:
            res = {"fri-kb-2^23": run_fri, "serving": run_serving, "quotient-kb-2^20": run_quotient}[args.workload](args)
            print(json.dumps(res), flush=True)
        return
    wl = WORKLOADS[args.workload]

    if args.impl == "reference":
        if rank == 0:
            ref = run_cpu(wl["shapes"](), wl["field"], wl["log_blowup"], wl["seed"], args.steps, args.warmup,
                          args.cpu_cells)
            line = {
                "metric": METRIC, "value": ref["value"], "unit": UNIT, "impl": "reference", "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ref["seconds_per_run"] * 1e3,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
                "data": "synthetic: seeded uniform field elements",
                "config": {"workload": args.workload, "sample": ref["sample"]},
                "cpu_baseline": {"value": ref["value"], "unit": UNIT, "cores": ref["cores"], "kind": "port",
                                 "cpu_model": ref["cpu_model"], "sample": ref["sample"]},
                "e2e": {"value": ref["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "note": "the reference's Rust/Plonky3 CPU path cannot be built here (no cargo, Plonky3 not "
                        "vendored); this is the C + OpenMP restatement (oracle) on all host threads",
            }
            print(json.dumps(line), flush=True)
        return

    result, shapes, field, b = run_gpu(args, rank, world, local)
    if rank == 0:
        if not args.skip_cpu:
            cpu = run_cpu(shapes, field, b, WORKLOADS[args.workload]["seed"], args.cpu_runs, 1, args.cpu_cells)
            result["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": cpu["cores"], "kind": "port",
                                      "cpu_model": cpu["cpu_model"], "sample": cpu["sample"]}
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
