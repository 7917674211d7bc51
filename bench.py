#!/usr/bin/env python
"""Benchmark: batched forward+backward GCUPS of the B200 search path.

Workload (one "step"): a batch of synthetic DNA reads, both strands, scored
against 64 synthetic profile HMMs (M log-uniform in [50, 800]; reads L
log-uniform in [150, 3000] nt, GC 0.4-0.6, 10% with implanted frameshifted
homologs) -- every (record, profile) pair, backward + forward with the
mid-anchored score, as one call of dmst_score_pairs (one persistent launch per
rows-per-lane group).  A cell is one (i, j), i in [0, M], j in [0, L), of one
pair; GCUPS = cells / s / 1e9.

Printed: one JSON line (rank 0).
  value      device-timed GCUPS with the reads resident in HBM (CUDA events on
             the library's stream around exactly --steps calls, max over ranks)
  e2e        the same metric through the public API with host buffers: each
             step copies its 2-bit packed reads host->device, decodes them on
             the device, scores, and copies the results back
  roofline   the dominant kernel (the R=4 mid kernel) against the FP32 issue
             peak: 52 algorithmic flops per cell (24 backward + 28 forward with
             the mid product) over its CUDA-event-timed duration
  plain      the same pairs (a sample) through the plain schedule, one pair per
             launch, and the batched/plain ratio
  cpu_baseline  the reference engine itself (oracle/_ref, compiled from the
             reference sources) on a bounded sample of the same pairs, all host
             threads
With --impl reference the reference engine alone runs (rank 0 only) and prints
the same line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from datetime import timedelta

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FLOPS_PER_CELL = 52  # 24 backward + 28 forward with the mid product
# adjoint, FP64 flops per cell counted from csrc/dp_adjoint.cuh: the forward
# recurrence with the T sum 24, the backward recurrence 21 and the gradient
# sums 22 (the checkpointed variant's forward recompute, 24 more, is not
# algorithmic work)
AG_FLOPS_PER_CELL = 67
SEARCH_E = 10.0                     # -e and the filter E-value by default (dummest-core.hh:60, dummest.cc:297-298)
FILTER_FLOPS_PER_CELL = 25          # the float filter: backward only
METRIC = "fwd+bwd GCUPS (batched persistent kernel)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--reads-per-step", type=int, default=5000,
                    help="reads per step (x2 strands x --profiles pairs); 20 steps of 5,000 reads are the "
                         "batched configuration's 100,000 reads")
    ap.add_argument("--parity-pairs", type=int, default=512,
                    help="pairs of the timed steps re-scored by the reference engine after the timed region "
                         "(0: none)")
    ap.add_argument("--profiles", type=int, default=64)
    ap.add_argument("--seed", type=int, default=20261205)
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-pairs", type=int, default=48)
    ap.add_argument("--rows-per-lane", type=int, default=0)
    ap.add_argument("--mmin", type=int, default=50,
                    help="batched workload: shortest profile (M log-uniform from here to --mmax)")
    ap.add_argument("--lmin", type=int, default=150,
                    help="batched workload: shortest read (L log-uniform from here to --lmax)")
    ap.add_argument("--mmax", type=int, default=800,
                    help="batched workload: longest profile (M log-uniform from 50; smaller cases for profiling)")
    ap.add_argument("--lmax", type=int, default=3000,
                    help="longest read of the batched workload (3000 in the stated configuration; smaller "
                         "values only to keep a profiling capture's device memory small)")
    ap.add_argument("--workload", choices=["batched", "genome", "autograd", "search", "align", "windows",
                                           "calibration"],
                    default="batched",
                    help="batched: 64 profiles x reads (the headline); genome: one M=2000 profile against a "
                         "10 Mbp genome in 10 kb windows; autograd: log-likelihood + gradient of an M=400 "
                         "profile over 4096 implant reads (L 600-2400), one SGD step per step; search: the "
                         "batched pairs through the two-wave search (filter, then mid on survivors); align: "
                         "the hit path with its traceback (an M=400 profile against homolog-carrying reads, "
                         "both strands, the hits' alignments traced); windows: the prefilter's hit windows "
                         "cut from a resident 256 Mbp genome and decoded on the device; calibration: the Gumbel "
                         "calibration batch, 500 profiles (M uniform 50-1500) x 200 i.i.d. uniform ACGT "
                         "sequences of 3000 nt each, mid scores and the FP64 fits")
    ap.add_argument("--cal-profiles", type=int, default=500, help="calibration workload: profiles")
    ap.add_argument("--cal-trials", type=int, default=200, help="calibration workload: sequences per profile")
    ap.add_argument("--cal-len", type=int, default=3000, help="calibration workload: sequence length")
    ap.add_argument("--win-mbp", type=int, default=256, help="windows workload: genome size (Mbp)")
    ap.add_argument("--win-hits", type=int, default=60000, help="windows workload: hit rows per step")
    ap.add_argument("--al-reads", type=int, default=256, help="align workload: reads per step (x2 strands)")
    ap.add_argument("--al-m", type=int, default=400, help="align workload: profile length")
    ap.add_argument("--al-gate", type=float, default=1e6, help="align workload: minProbRatio of every pair")
    ap.add_argument("--ag-reads", type=int, default=4096, help="autograd workload: reads per rank")
    ap.add_argument("--ag-m", type=int, default=400, help="autograd workload: profile length")
    ap.add_argument("--ag-lmin", type=int, default=600, help="autograd workload: shortest read")
    ap.add_argument("--ag-lmax", type=int, default=2400, help="autograd workload: longest read")
    ap.add_argument("--ag-ckpt", choices=["on", "off", "auto"], default="on",
                    help="autograd workload: the adjoint's column checkpointing (every 64 columns)")
    ap.add_argument("--no-autotune", action="store_true", help="skip the kernel-shape autotuner")
    ap.add_argument("--no-graph", action="store_true", help="direct launches instead of CUDA-graph replay")
    ap.add_argument("--no-async", action="store_true", help="synchronous calls (no submit/complete overlap)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU, weak scaling: every rank scores
# its own reads against all profiles; no data-path collective)
# ---------------------------------------------------------------------------
def dist_env():
    """(rank, world, local rank) from the launcher's environment (torchrun)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def dist_setup(backend: str = "nccl"):
    """One process per GPU; a short process-group timeout so that ranks that
    wait for a missing peer end with an error instead of hanging."""
    rank, world, local = dist_env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return rank, world, local


def _reduce(x: float, world: int, op: str) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x: float, world: int) -> float:
    return _reduce(x, world, "max")


def allreduce_sum(x: float, world: int) -> float:
    return _reduce(x, world, "sum")


def rank_seed(seed: int, rank: int) -> int:
    """Each rank scores its own reads (weak scaling: pairs shard by rank)."""
    return seed + 1 + 1000 * rank


def aggregate(cells: float, ms: float, world: int) -> tuple[float, float, float]:
    """Whole-job throughput: the cells of all ranks over the slowest rank's
    device time.  Returns (GCUPS, max ms, total cells)."""
    ms_max = allreduce_max(ms, world)
    cells_all = allreduce_sum(cells, world)
    return cells_all / (ms_max * 1e-3) / 1e9, ms_max, cells_all


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
def workload_config(args, world: int) -> dict:
    """The workload both arms report (cells_per_step is added by the GPU arm,
    which counts them)."""
    if args.workload == "autograd":
        return {
            "workload": f"log-likelihood + gradient (adjoint, FP64): 1 profile M={args.ag_m} x {args.ag_reads} "
                        f"reads L uniform {args.ag_lmin}-{args.ag_lmax} nt, each carrying a frameshifted homolog, "
                        "one SGD step of the emission/transition/frameshift logits per step; column "
                        f"checkpointing every 64 nt: {args.ag_ckpt}",
            "profiles": 1, "pairs_per_step": args.ag_reads, "l2": "inputs larger than L2 (forward store)",
            "parallelism": f"replicas x{world} (reads sharded per rank)",
        }
    if args.workload == "search":
        return {
            "workload": f"two-wave search (float filter on every pair, mid-anchored score on survivors, E <= "
                        f"{SEARCH_E:g}): {args.profiles} profiles M log-uniform {args.mmin}-{args.mmax} x reads L "
                        f"log-uniform {args.lmin}-{args.lmax} nt, GC 0.4-0.6, 10% implants, both strands; gates from each profile's "
                        "calibration (200 x 3 kb random sequences)",
            "reads_per_step": args.reads_per_step, "records_per_step": 2 * args.reads_per_step,
            "profiles": args.profiles, "pairs_per_step": 2 * args.reads_per_step * args.profiles,
            "l2": "inputs larger than L2 (W1 slots)",
            "parallelism": f"replicas x{world} (pairs sharded per rank)",
        }
    if args.workload == "align":
        return {
            "workload": f"hit path with traceback (findSimilarities needAlign): 1 profile M={args.al_m} x "
                        f"{args.al_reads} reads (a frameshifted homolog of the whole profile between two 500 nt "
                        f"random flanks), both strands, minProbRatio {args.al_gate:g}: every pair scored, the "
                        "hits' alignments traced",
            "profiles": 1, "reads_per_step": args.al_reads, "pairs_per_step": 2 * args.al_reads,
            "l2": "inputs larger than L2 (traceback tables)",
            "parallelism": f"replicas x{world} (reads sharded per rank)",
        }
    if args.workload == "windows":
        return {
            "workload": f"prefilter window stage: {args.win_hits} six-frame BLAST-tab hit rows of 8 profiles (M "
                        f"log-uniform 100-800) on a {args.win_mbp} Mbp synthetic genome (64 records, GC 0.45, 1% "
                        "lower case, N runs) -> merged windows (+-3M nt around each hit, both strands) -> "
                        "codon codes of every window contig on the device",
            "profiles": 8, "hits_per_step": args.win_hits,
            "l2": "each step a different window set (codes written > L2); L2 flushed (256 MB) before each "
                  "kernel-timed launch",
            "parallelism": f"replicas x{world} (one genome per rank)",
        }
    if args.workload == "calibration":
        return {
            "workload": f"Gumbel calibration batch: {args.cal_profiles} profiles M uniform 50-1500 x "
                        f"{args.cal_trials} i.i.d. uniform ACGT sequences of {args.cal_len} nt per profile, mid "
                        "scores (fwd+bwd) in one call, lambda/K fitted on the host in FP64 (estimateGumbel)",
            "profiles": args.cal_profiles, "pairs_per_step": args.cal_profiles * args.cal_trials,
            "l2": "inputs larger than L2 (W1 slots)",
            "parallelism": f"replicas x{world}",
        }
    if args.workload == "genome":
        return {
            "workload": "long-profile genome scan: 1 profile M=2000 x a 10 Mbp synthetic genome (GC 0.45, "
                        "200 implanted frameshifted homologs) in 10 kb windows overlapping 1 kb, both strands",
            "profiles": 1, "pairs_per_step": 2222, "l2": "inputs larger than L2 (W1 slots)",
            "parallelism": f"replicas x{world} (one genome per rank)",
        }
    return {
        "workload": f"batched fwd+bwd (mid-anchored score): {args.profiles} profiles M log-uniform {args.mmin}-{args.mmax} x "
                    f"reads L log-uniform {args.lmin}-{args.lmax} nt, GC 0.4-0.6, 10% implants, both strands",
        "reads_per_step": args.reads_per_step, "records_per_step": 2 * args.reads_per_step,
        "profiles": args.profiles, "pairs_per_step": 2 * args.reads_per_step * args.profiles,
        "l2": "inputs larger than L2 (W1 slots)",
        "parallelism": f"replicas x{world} (pairs sharded per rank)",
    }


def make_profiles(seed, n, mmax=800, mmin=50):
    from dummest_b200 import synth
    rng = np.random.default_rng(seed)
    Ms = np.exp(rng.uniform(np.log(mmin), np.log(mmax), size=n)).round().astype(int)
    profiles = [synth.make_profile(rng, int(M), f"synth{k:03d}") for k, M in enumerate(Ms)]
    return profiles, synth.hmmer3_text(profiles)


def make_workload(args, rank: int, n_steps: int, world: int = 0):
    """(profiles, HMMER3 text, steps): each step a list of records scored
    against every profile.  With world >= 1 (the batched workload sharded
    over `world` ranks) every rank builds the same read sets, world x
    reads_per_step reads each: n_steps distinct sets at one rank, else enough
    to cover the configuration's 100,000 reads (the steps cycle through
    them); world = 0 gives each rank its own reads."""
    if args.workload == "genome":
        from dummest_b200 import synth
        prof, windows = synth.genome_scan_config(seed=rank_seed(args.seed, rank))
        return [prof], synth.hmmer3_text([prof]), [windows] * (1 if world >= 1 else n_steps)
    if args.workload == "align":
        from dummest_b200 import synth
        rng = np.random.default_rng(args.seed)
        prof = synth.make_profile(rng, args.al_m, "align")
        rng = np.random.default_rng(rank_seed(args.seed, rank))
        steps = []
        for _ in range(n_steps):
            reads = [synth.random_dna(rng, 500) + synth.sample_homolog(rng, prof, args.al_m, fs_rate=0.01)
                     + synth.random_dna(rng, 500) for _ in range(args.al_reads)]
            steps.append(synth.both_strands(reads))
        return [prof], synth.hmmer3_text([prof]), steps
    profiles, txt = make_profiles(args.seed, args.profiles, args.mmax, args.mmin)
    if world >= 1:
        per = world * args.reads_per_step
        n_sets = n_steps if world == 1 else min(n_steps, args.warmup + -(-100_000 // per))
        return profiles, txt, make_steps(rank_seed(args.seed, 0), profiles, n_sets, per, args.lmax, args.lmin)
    return profiles, txt, make_steps(rank_seed(args.seed, rank), profiles, n_steps, args.reads_per_step, args.lmax,
                                     args.lmin)


def make_steps(seed, profiles, n_steps, reads_per_step, lmax=3000, lmin=150):
    from dummest_b200 import synth
    rng = np.random.default_rng(seed)
    steps = []
    for _ in range(n_steps):
        reads = synth.make_reads(rng, reads_per_step, lmin, lmax, profiles, 0.10, gc_range=(0.4, 0.6))
        steps.append(synth.both_strands(reads))
    return steps


from dummest_b200.shards import PAIR_DTYPE, RESULT_DTYPE  # noqa: E402


def pair_array(sids, pids, min_prob_ratio=-2.0):
    """Every (profile, record) pair, profile-major, as a ctypes dmst_pair
    array backed by numpy (the pair of profile index a and record index b is
    element a * len(sids) + b)."""
    from dummest_b200 import _ffi as F
    assert F.C.sizeof(F.Pair) == PAIR_DTYPE.itemsize
    sids = np.asarray(sids, np.int32)
    pids = np.asarray(pids, np.int32)
    arr = np.empty(len(sids) * len(pids), PAIR_DTYPE)
    arr["seq"] = np.tile(sids, len(pids))
    arr["profile"] = np.repeat(pids, len(sids))
    arr["min_prob_ratio"] = min_prob_ratio
    out = (F.Pair * len(arr)).from_buffer(arr)
    out._keep = arr  # the ctypes array views arr's memory
    return out


def result_view(res) -> np.ndarray:
    """A ctypes dmst_result array as a numpy structured array (no copy);
    numpy result arrays pass through."""
    from dummest_b200 import _ffi as F
    if isinstance(res, np.ndarray):
        return res
    assert F.C.sizeof(F.Result) == RESULT_DTYPE.itemsize
    return np.frombuffer(res, dtype=RESULT_DTYPE)


def parity_sample(hmm_text, checked_steps, n_sample, seed):
    """Scores a seeded sample of timed pairs with the reference engine
    (oracle/_ref, FP32 findSimilarities needAlign=false) and compares them
    with the results the timed calls returned: mid and filter ExpScores bit
    for bit.  checked_steps: (records, results) of timed steps, results in
    profile-major pair order.  The sample holds n_sample random pairs plus,
    for every step, its longest record against its longest profile."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.ref import RefEngine, available
    if not available(32):
        return {"checked": 0, "bit_equal": 0, "max_abs_bits": None, "note": "oracle/_ref not built"}
    e = RefEngine(32)
    e.set_rates()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(hmm_text)
        path = f.name
    n_prof = e.load_profiles(path)
    os.unlink(path)
    Ms = np.array([e.profile(p)[1].shape[0] - 1 for p in range(n_prof)])
    rng = np.random.default_rng(seed + 77)
    picks = set()
    for i, (recs, _) in enumerate(checked_steps):
        picks.add((i, int(np.argmax(Ms)), int(np.argmax([len(r) for r in recs]))))
    while len(picks) < n_sample + len(checked_steps):
        i = int(rng.integers(0, len(checked_steps)))
        picks.add((i, int(rng.integers(0, n_prof)), int(rng.integers(0, len(checked_steps[i][0])))))
    by_prof = {}
    for t in sorted(picks, key=lambda t: (t[1], t[0], t[2])):
        by_prof.setdefault(t[1], []).append(t)
    jobs = [(p, lst[b:b + e.width]) for p, lst in by_prof.items() for b in range(0, len(lst), e.width)]

    def run(job):
        p, lst = job
        codes = [e.decode(e.encode(checked_steps[i][0][r])) for i, _, r in lst]
        return job, e.find_similarities(p, codes)

    t0 = time.perf_counter()
    checked = equal = 0
    worst, cells, largest = 0.0, 0.0, (0, 0)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        for (p, lst), refs in ex.map(run, jobs):
            for (i, _, r), (mm, me, ml, fm, fe) in zip(lst, refs):
                recs, res = checked_steps[i]
                got = result_view(res)[p * len(recs) + r]
                same = (np.float32(got["mid_m"]) == np.float32(mm) and int(got["mid_e"]) == me
                        and np.float32(got["flt_m"]) == np.float32(fm) and int(got["flt_e"]) == fe)
                checked += 1
                equal += int(same)
                if np.isfinite(ml) and np.isfinite(got["mid_ln"]):
                    worst = max(worst, abs(float(got["mid_ln"]) - ml) / np.log(2.0))
                elif not (np.isinf(ml) and np.isinf(got["mid_ln"])):
                    worst = float("inf")
                cells += (Ms[p] + 1) * len(recs[r])
                largest = max(largest, (int(Ms[p]), len(recs[r])))
    lmax = max(len(r) for recs, _ in checked_steps for r in recs)
    return {"checked": checked, "bit_equal": equal, "max_abs_bits": worst,
            "sample": f"{n_sample} seeded random pairs of {len(checked_steps)} timed steps (every 4th) plus each "
                      f"step's longest record x longest profile (M={largest[0]}, L up to {lmax}); "
                      f"{cells:.3e} cells, reference FP32 engine, {time.perf_counter() - t0:.1f} s",
            "compared": "mid and filter ExpScore (mantissa, exponent) of the timed calls' results"}


# ---------------------------------------------------------------------------
# GPU clock sampling during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.device)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_model() -> str:
    """The host CPU's model name and logical CPU count (from /proc/cpuinfo)."""
    try:
        names = [ln.split(":", 1)[1].strip() for ln in open("/proc/cpuinfo") if ln.startswith("model name")]
        return f"{names[0]} ({len(names)} logical CPUs)" if names else "unknown"
    except OSError:
        return "unknown"


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        return {}


def traffic_per_cell():
    """DRAM bytes per cell of the mid kernel from the committed ncu summary."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "dpKernel_stagger_640000pairs_traffic.json")))["dram_bytes_per_cell"]
    except (OSError, KeyError, ValueError):
        return None


# ---------------------------------------------------------------------------
# CPU baseline: the reference engine (oracle/_ref) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_baseline(hmm_text, records, n_profiles, seconds, seed):
    from oracle.ref import RefEngine, available
    if not available(32):
        return None
    e = RefEngine(32)
    e.set_rates()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(hmm_text)
        path = f.name
    n = e.load_profiles(path)
    os.unlink(path)
    Ms = [e.profile(p)[1].shape[0] for p in range(n)]  # M+1 rows
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    codes = [e.decode(e.encode(r)) for r in records]
    lens = np.array([len(c) for c in codes], dtype=np.float64)
    # Every record of the step against profiles in random order until the time
    # budget is spent: each call hands the reference >= 8 x threads lanes, so
    # all threads have SIMD batches to run.
    # Blocks of records (all of them, or 32 SIMD batches per thread when a
    # step has few profiles) against profiles in random order until the time
    # budget is spent; each call hands every thread SIMD batches to run.
    block = len(codes) if n > 4 else min(len(codes), 32 * 8 * threads)
    done_cells, done_s, used, recs = 0.0, 0.0, 0, 0
    for p in rng.permutation(n):
        for b0 in range(0, len(codes), block):
            t = time.perf_counter()
            e.score_many(int(p), codes[b0:b0 + block], threads=threads, mode=0)
            done_s += time.perf_counter() - t
            done_cells += Ms[p] * lens[b0:b0 + block].sum()
            recs += min(block, len(codes) - b0)
            if done_s >= seconds:
                break
        used += 1
        if done_s >= seconds:
            break
    return {
        "value": done_cells / done_s / 1e9,
        "unit": "GCUPS",
        "cores": threads, "cpu_model": cpu_model(),
        "kind": "reference",
        "sample": f"{recs} record-profile pairs of one step ({used} of {n} profiles), "
                  f"{done_cells:.3e} cells in {done_s:.1f} s, reference FP32 engine "
                  "(findSimilarities needAlign=false, the calibration call) in <=8-lane SIMD batches",
    }


# ---------------------------------------------------------------------------
def search_gates(fits, total_length):
    """Per-profile float gates of the filter wave (dmst_filter_threshold)."""
    import dummest_b200 as d
    return np.array([d.filter_threshold(f["lambda_filter"], f["K_filter"], total_length, SEARCH_E) for f in fits],
                    np.float32)


def cpu_search_baseline(hmm_text, records, gates, seconds, seed):
    """The reference engine's two waves on a bounded sample: its float filter
    (findSimilaritiesBackwardOnly) on every record x profile, then its mid
    score (findSimilarities) on the survivors, all host threads."""
    from oracle.ref import RefEngine, available
    if not available(32):
        return None
    e = RefEngine(32)
    e.set_rates()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(hmm_text)
        path = f.name
    n = e.load_profiles(path)
    os.unlink(path)
    Ms = [e.profile(p)[1].shape[0] for p in range(n)]
    threads = os.cpu_count() or 1
    rng = np.random.default_rng(seed)
    codes = [e.decode(e.encode(r)) for r in records]
    lens = np.array([len(c) for c in codes], dtype=np.float64)
    done_cells, done_s, used, surv = 0.0, 0.0, 0, 0
    for p in rng.permutation(n):
        t = time.perf_counter()
        # mode 1 gives log((double)best); b >= gate (floats) <=> log b >= log gate
        _, flt = e.score_many(int(p), codes, threads=threads, mode=1)
        lg = np.log(np.float64(gates[p]))
        keep = [k for k, lb in enumerate(flt) if lb > -np.inf and (lb >= lg or lb == np.inf)]
        if keep:
            e.score_many(int(p), [codes[k] for k in keep], threads=threads, mode=0)
        done_s += time.perf_counter() - t
        done_cells += Ms[p] * lens.sum()
        surv += len(keep)
        used += 1
        if done_s >= seconds:
            break
    return {"value": done_cells / done_s / 1e9, "unit": "GCUPS", "cores": threads, "cpu_model": cpu_model(), "kind": "reference",
            "sample": f"{used} of {n} profiles x {len(codes)} records of one step ({surv} survivors), "
                      f"{done_cells:.3e} cells in {done_s:.1f} s: the reference's float filter on every pair, "
                      "then its mid score on the survivors"}


def cpu_align_baseline(hmm_text, records, gate, seconds):
    """The reference's hit path with its traceback (findSimilarities with
    needAlign, oracle/_ref) on the box's cores: 8-record SIMD batches of the
    step, one per thread at a time, until the time budget is spent."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle.ref import RefEngine, available
    if not available(32):
        return None
    e = RefEngine(32)
    e.set_rates()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(hmm_text)
        path = f.name
    e.load_profiles(path)
    os.unlink(path)
    M1 = e.profile(0)[1].shape[0]
    codes = [e.decode(e.encode(r)) for r in records]
    threads = os.cpu_count() or 1
    batches = [codes[b:b + 8] for b in range(0, len(codes), 8)]
    done_cells, done_b, t0 = 0.0, 0, time.perf_counter()
    with ThreadPoolExecutor(threads) as pool:
        while time.perf_counter() - t0 < seconds and done_b < len(batches):
            chunk = batches[done_b:done_b + threads]
            list(pool.map(lambda b: e.align(0, b, [gate] * len(b)), chunk))
            done_b += len(chunk)
            done_cells += M1 * sum(len(c) for b in chunk for c in b)
    dt = time.perf_counter() - t0
    return {"value": done_cells / dt / 1e9, "unit": "GCUPS", "cores": threads, "cpu_model": cpu_model(), "kind": "reference",
            "sample": f"{done_b} 8-record batches of one step ({done_cells:.3e} cells) in {dt:.1f} s, reference "
                      "FP32 engine, findSimilarities with needAlign (scores, anchors, traceback)"}


def run_align(args, rank, world, local):
    import dummest_b200 as d
    from dummest_b200 import _ffi as F
    import torch

    n_steps = args.warmup + args.steps
    profiles, txt, steps = make_workload(args, rank, n_steps)
    ctx = d.Context(device=local)
    pid = ctx.load_hmm(txt)[0]
    M = ctx.profile_length(pid)

    def pairs_for(sids):
        arr = (F.Pair * len(sids))()
        for k, s in enumerate(sids):
            arr[k].seq, arr[k].profile, arr[k].min_prob_ratio = s, pid, args.al_gate
        return arr

    step_pairs = [pairs_for(ctx.add_dna(recs)) for recs in steps]
    cells_step = [float(sum(len(r) for r in recs)) * (M + 1) for recs in steps]
    for w in range(args.warmup):
        ctx.align_raw(step_pairs[w])
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    cells, exact_ms, outs = 0.0, 0.0, []
    phases = {}
    for k in range(args.warmup, n_steps):
        outs.append(ctx.align_raw(step_pairs[k]))
        exact_ms += ctx.last_timing()["exact_ms"]  # the traced hits' exact replay
        for key, v in ctx.last_align_timing().items():
            phases[key] = phases.get(key, 0.0) + v
        cells += cells_step[k]
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    value, ms_max, cells_all = aggregate(cells, ms, world)
    n_al = n_seg = 0
    hit_cells = 0.0
    for k, (al, sg) in zip(range(args.warmup, n_steps), outs):
        hits = {a.pair for a in al}
        hit_cells += sum(len(steps[k][i]) * (M + 1) for i in hits)
        n_al += len(al)
        n_seg += len(sg)
    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = n_sm * 128 * 2 * sm_max * 1e6 / 1e12
    # the exact replay of the hits: discovery and replay sweeps in both directions
    achieved = 2 * FLOPS_PER_CELL * hit_cells / (exact_ms / 1e3) / 1e12 if exact_ms > 0 else None
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak if achieved else None, "traffic": None,
                "peak_source": f"derived: {n_sm} SMs x 128 FP32 lanes x 2 x sm_max_mhz {sm_max:g}",
                "kernel": "the exact kernel's discovery + replay sweeps with the traceback stores, over the hits",
                "algorithmic_flops_per_cell": 2 * FLOPS_PER_CELL}
    # e2e: each step's reads copied (2-bit packed) and decoded, the call, its alignments copied back
    packed = [d.pack_dna(recs) for recs in steps]
    ctx.clear_sequences()
    base, e2e_pairs = 0, []
    for k in range(n_steps):
        e2e_pairs.append(pairs_for(list(range(base, base + len(steps[k])))))
        base += len(steps[k])
    for w in range(args.warmup):
        words, mask, lens = packed[w]
        ctx.add_packed(words, lens, mask)
        ctx.align_raw(e2e_pairs[w])
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for k in range(args.warmup, n_steps):
        words, mask, lens = packed[k]
        ctx.add_packed(words, lens, mask)
        al, sg = ctx.align_raw(e2e_pairs[k])
        h2d += words.nbytes + mask.nbytes + 12 * len(lens) + 12 * len(e2e_pairs[k])
        d2h += 40 * len(al) + 12 * len(sg)
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d // args.steps,
           "d2h_bytes_per_step": d2h // args.steps}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_align_baseline(txt, steps[args.warmup], args.al_gate, args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": "hit-path traceback GCUPS (cells of every pair; hits traced)", "value": value, "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args, world), cells_per_step=cells / args.steps),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk,
            "gpu_launches": int(phases.get("launches", 0)), "alignments_per_step": n_al / args.steps, "segments_per_step": n_seg / args.steps,
            "hit_cell_fraction": hit_cells / cells, "exact_ms_per_step": exact_ms / args.steps,
            "phases_ms_per_step": {k: v / args.steps for k, v in phases.items() if k != "launches"}}), flush=True)
    ctx.close()


# ---------------------------------------------------------------------------
# the prefilter window stage: hit rows -> windows -> sequences on the device
# ---------------------------------------------------------------------------
WIN_BYTES_PER_NT = 1.375  # per window nt: its code written (1 B) + its base read (2 bits + 1 mask bit)


def windows_problem(args, rank):
    """(genome FASTA text, record names, record lengths, profile names,
    profile lengths, hit texts per step)."""
    rng = np.random.default_rng(rank_seed(args.seed, rank))
    n_rec = 64
    per = args.win_mbp * 1_000_000 // n_rec
    names = [f"chr{k + 1}" for k in range(n_rec)]
    parts = []
    for name in names:
        seq = rng.choice(np.frombuffer(b"ACGT", np.uint8), size=per, p=[0.275, 0.225, 0.225, 0.275])
        seq[rng.random(per) < 0.01] += 32
        for _ in range(4):
            a = int(rng.integers(0, per - 200))
            seq[a:a + int(rng.integers(1, 200))] = ord("N")
        rows = per // 60
        body = np.full((rows, 61), ord("\n"), np.uint8)
        body[:, :60] = seq[:rows * 60].reshape(rows, 60)
        parts.append(b">" + name.encode() + b"\n" + body.tobytes() + seq[rows * 60:].tobytes() + b"\n")
    genome = b"".join(parts)
    Ms = np.exp(rng.uniform(np.log(100), np.log(800), size=8)).round().astype(int)
    pnames = [f"PF{k:05d}.1" for k in range(8)]
    frames = np.array([1, 2, 3, -1, -2, -3])
    steps = []
    for _ in range(args.warmup + args.steps):
        r = rng.integers(0, n_rec, args.win_hits)
        q = rng.integers(0, 8, args.win_hits)
        f = frames[rng.integers(0, 6, args.win_hits)]
        c = rng.integers(1, per // 3 - 1, args.win_hits)
        h = rng.integers(0, 60, args.win_hits)
        lines = [f"{pnames[q[k]]}\t{names[r[k]]}_frame={f[k]:+d}\t45.0\t90\t10\t1\t1\t30\t{max(1, c[k] - h[k])}"
                 f"\t{c[k] + h[k]}\t1e-10\t55.0\n" for k in range(args.win_hits)]
        steps.append("".join(lines).encode())
    return genome, names, [per] * n_rec, pnames, Ms.tolist(), steps


def cpu_windows_baseline(genome, windows, names, seconds):
    """The engine side of the pipeline's text path on the host: the windowed
    FASTA (bedtools getfasta -s, restated, not timed) read and decoded by the
    reference's own code (readContig + decodeSequence of its PIPELINE_MODE
    build, oracle/_ref: dmstref_read_decode), chunks of 64 windows on every host
    thread (the ctypes call releases the interpreter lock), until the sample
    time is spent."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import windows as W
    from oracle import ref as R
    recs = W.fasta_records(genome)
    texts = []
    for w in windows[:8192]:
        name = names[w.record].encode()
        seq = recs[name][w.start:w.end]
        if w.strand < 0:
            seq = seq.translate(W._COMP)[::-1]
        texts.append(b">%s/%d-%d length=%d profile=P %s\n%s\n" % (
            name, w.start + 1, w.end, len(recs[name]), b"plus_strand" if w.strand > 0 else b"minus_strand_revcomp",
            seq))
    chunks = [b"".join(texts[k:k + 64]) for k in range(0, len(texts), 64)]
    R.read_decode(chunks[0])  # the harness's one-time set-up, before the threads
    threads = os.cpu_count() or 1
    nt, done, t0 = 0, 0, time.perf_counter()
    with ThreadPoolExecutor(threads) as pool:
        while time.perf_counter() - t0 < seconds:
            batch = [chunks[(done + j) % len(chunks)] for j in range(4 * threads)]
            nt += sum(n for n, _ in pool.map(R.read_decode, batch))
            done += len(batch)
    dt = time.perf_counter() - t0
    return {"value": nt / dt / 1e9, "unit": "Gnt/s", "cores": threads, "cpu_model": cpu_model(), "kind": "reference",
            "sample": f"{done} chunks of 64 windowed FASTA records ({nt} nt; the first {len(texts)} windows, "
                      f"cycled) for {dt:.1f} s: the reference's readContig + decodeSequence (PIPELINE_MODE build, "
                      f"oracle/_ref), {threads} threads; bedtools getfasta's own time not counted"}


def run_windows(args, rank, world, local):
    import dummest_b200 as d
    from dummest_b200 import _ffi as F
    import torch

    genome, names, lens, pnames, plens, steps = windows_problem(args, rank)
    ctx = d.Context(device=local)
    ctx.genome_load(genome)
    wins = [d.windows_from_hits(h, names, lens, pnames, plens)[0] for h in steps]
    cap = [len(w) * 4 + 16 for w in wins]
    outs = [(F.Contig * c)() for c in cap]
    n_steps = args.warmup + args.steps
    for k in list(range(n_steps)) + list(range(args.warmup)):  # device buffers sized for every step first
        ctx.clear_sequences()
        ctx.add_windows_raw(wins[k], outs[k])
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    counts = []
    for k in range(args.warmup, n_steps):
        ctx.clear_sequences()  # host bookkeeping only: the step's codes reuse the same device space
        counts.append(ctx.add_windows_raw(wins[k], outs[k]))
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    nt = 0
    for k, n in zip(range(args.warmup, n_steps), counts):
        nt += sum(c.length for c in outs[k][:n] if c.seq_id >= 0)
    nt_all = allreduce_sum(float(nt), world)
    ms_max = allreduce_max(ms, world)
    value = nt_all / (ms_max / 1e3) / 1e9
    # the decode kernel alone, one launch per step, L2 flushed before each
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    kern_ms = 0.0
    for k in range(args.warmup, n_steps):
        flush.fill_(k & 0xFF)
        torch.cuda.synchronize()
        ctx.clear_sequences()
        ctx.add_windows_raw(wins[k], outs[k])
        kern_ms += ctx.last_windows_ms()
    peaks = measured_peaks()
    hbm = peaks.get("hbm_gbs", 6451.2)
    achieved = WIN_BYTES_PER_NT * nt / (kern_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": None, "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)",
                "kernel": "windowDecodeKernel, CUDA events on the library stream around each launch",
                "algorithmic_bytes_per_nt": WIN_BYTES_PER_NT, "kernel_ms_per_step": kern_ms / args.steps}
    # e2e: from each step's hit rows in host memory: the windows (host), the
    # contigs (host), the segment descriptors up and the decode on the device
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    added = []
    for k in range(args.warmup, n_steps):
        w, _, _ = d.windows_from_hits(steps[k], names, lens, pnames, plens)
        ctx.clear_sequences()
        added.append(ctx.add_windows_raw(w, outs[k]))
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    # one upload per step (counted after the timed region): a 40-byte
    # descriptor per sequence, then one int per decode block of 256 chunks of
    # 16 nt (the contig of the block's first chunk).  The upload is a pageable
    # copy, so it waits for the library stream; that wait is inside e2e.
    h2d = 0
    for k, n in zip(range(args.warmup, n_steps), added):
        seqs = [c for c in outs[k][:n] if c.seq_id >= 0]
        chunks = sum((c.length + 15) // 16 for c in seqs)
        h2d += 40 * len(seqs) + 4 * ((chunks + 255) // 256)
    e2e = {"value": nt_all / e2e_s / 1e9, "unit": "Gnt/s", "h2d_bytes_per_step": h2d // args.steps,
           "d2h_bytes_per_step": 0,
           "note": "the step's result (contigs, sequence ids) is host memory; the codes stay on the device"}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_windows_baseline(genome, wins[args.warmup], names, args.cpu_seconds)
    if rank == 0:
        print(json.dumps({
            "metric": "prefilter window stage: window nt decoded per second", "value": value, "unit": "Gnt/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": dict(workload_config(args, world), windows_per_step=sum(len(wins[k]) for k in
                           range(args.warmup, n_steps)) / args.steps, nt_per_step=nt / args.steps),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "clocks": clk,
            "gpu_launches": args.steps}), flush=True)
    ctx.close()


def calibration_problem(args, rank):
    """(profiles, HMMER3 text, sequences) of the calibration batch: profile p
    is scored against sequences[p * trials : (p + 1) * trials]."""
    from dummest_b200 import synth
    rng = np.random.default_rng(rank_seed(args.seed + 3, rank))
    Ms = rng.integers(50, 1501, size=args.cal_profiles)
    profiles = [synth.make_profile(rng, int(M), f"cal{k:03d}") for k, M in enumerate(Ms)]
    seqs = [synth.random_dna(rng, args.cal_len, 0.5) for _ in range(args.cal_profiles * args.cal_trials)]
    return profiles, synth.hmmer3_text(profiles), seqs


def _ref_engine(hmm_text):
    from oracle.ref import RefEngine, available
    if not available(32):
        return None
    e = RefEngine(32)
    e.set_rates()
    with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
        f.write(hmm_text)
        path = f.name
    e.load_profiles(path)
    os.unlink(path)
    return e


def cpu_calibration_baseline(hmm_text, seqs, trials, seconds, seed):
    """The reference engine on a bounded sample of the calibration batch:
    whole profiles (their trials, findSimilarities needAlign=false on all
    host threads) in random order until the time budget is spent."""
    e = _ref_engine(hmm_text)
    if e is None:
        return None
    threads = os.cpu_count() or 1
    n = len(seqs) // trials
    Ms = [e.profile(p)[1].shape[0] for p in range(n)]
    rng = np.random.default_rng(seed)
    done_cells, done_s, used = 0.0, 0.0, 0
    for p in rng.permutation(n):
        codes = [e.decode(e.encode(s)) for s in seqs[p * trials:(p + 1) * trials]]
        t = time.perf_counter()
        e.score_many(int(p), codes, threads=threads, mode=0)
        done_s += time.perf_counter() - t
        done_cells += Ms[p] * float(sum(len(c) for c in codes))
        used += 1
        if done_s >= seconds:
            break
    return {"value": done_cells / done_s / 1e9, "unit": "GCUPS", "cores": threads, "cpu_model": cpu_model(),
            "kind": "reference",
            "sample": f"{used} of {n} profiles x {trials} sequences, {done_cells:.3e} cells in {done_s:.1f} s, "
                      "reference FP32 engine (the calibration call, findSimilarities needAlign=false)"}


def calibration_parity(hmm_text, seqs, trials, Ms, res, seq_len):
    """Three profiles of the batch (the longest, the median and the shortest)
    re-scored by the reference engine: trial ln-scores compared bit for bit,
    and the E-values of the two FP64 fits (estimateGumbel) compared over the
    range from the median score to 60 bits above it."""
    import dummest_b200 as d
    e = _ref_engine(hmm_text)
    if e is None:
        return None
    order = np.argsort(Ms, kind="stable")
    picks = sorted({int(order[-1]), int(order[len(order) // 2]), int(order[0])})
    checked = equal = 0
    worst_e = 0.0
    t0 = time.perf_counter()
    for p in picks:
        codes = [e.decode(e.encode(s)) for s in seqs[p * trials:(p + 1) * trials]]
        rm, rf = e.score_many(p, codes, threads=os.cpu_count() or 1, mode=0)
        got = res[p * trials:(p + 1) * trials]
        checked += 2 * trials
        equal += int(np.sum(got["mid_ln"] == rm)) + int(np.sum(got["flt_ln"] == rf))
        for ours, theirs in ((got["mid_ln"], rm), (got["flt_ln"], rf)):
            g, w = d.estimate_gumbel(ours, seq_len), e.estimate_gumbel(theirs, seq_len)
            s_nats = np.linspace(np.median(theirs), np.median(theirs) + 60 * np.log(2.0), 31)
            ratio = (g[1] * np.exp(-g[0] * s_nats)) / (w[1] * np.exp(-w[0] * s_nats))
            worst_e = max(worst_e, float(np.max(np.abs(ratio - 1.0))))
    return {"checked": checked, "bit_equal": equal, "max_evalue_rel_err": worst_e,
            "sample": f"profiles M={[int(Ms[p]) for p in picks]}, {trials} sequences each, mid and filter "
                      f"ln-scores; reference FP32 engine, {time.perf_counter() - t0:.1f} s"}


def run_calibration(args, rank, world, local):
    import dummest_b200 as d
    from dummest_b200 import _ffi as F
    import torch

    profiles, txt, seqs = calibration_problem(args, rank)
    T, n_steps = args.cal_trials, args.warmup + args.steps
    ctx = d.Context(device=local, rows_per_lane=args.rows_per_lane)
    pids = ctx.load_hmm(txt)
    Ms = np.array([ctx.profile_length(p) for p in pids])

    def pairs_for(sids):
        arr = np.zeros(len(sids), PAIR_DTYPE)
        arr["seq"] = sids
        arr["profile"] = np.repeat(np.asarray(pids, np.int32), T)
        arr["min_prob_ratio"] = -2.0
        out = (F.Pair * len(arr)).from_buffer(arr)
        out._keep = arr
        return out

    def fit_all(res):
        """FP64 lambda and K of every profile (mid, then filter scores)."""
        r = result_view(res)
        fits = np.zeros((len(pids), 4))
        for p in range(len(pids)):
            sl = slice(p * T, (p + 1) * T)
            fits[p, 0:2] = d.estimate_gumbel(r["mid_ln"][sl], args.cal_len)[:2]
            fits[p, 2:4] = d.estimate_gumbel(r["flt_ln"][sl], args.cal_len)[:2]
        return fits

    sids = ctx.add_dna(seqs)
    pairs = pairs_for(sids)
    cells = float(args.cal_len) * float((Ms + 1).sum()) * T
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    tuning = None
    if not args.no_autotune and args.rows_per_lane == 0:
        samp = [k for p in range(len(pids)) for k in range(p * T, p * T + 8)]
        rates = ctx.autotune([sids[k] for k in samp], [pids[k // T] for k in samp])
        tuning = {"gcups_computed_cells": {f"R{r}/W{w}": round(v, 2) for (r, w), v in rates.items()}}
    MODE = d.MODE_MID | (0 if args.no_graph else d.MODE_GRAPH)
    # warm-up steps in the timed steps' pattern (both call slots in use)
    for w in range(args.warmup):
        ctx.submit_raw(pairs, MODE)
        if w > 0:
            ctx.complete()
    if args.warmup:
        ctx.complete()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    launches, dp_ms, last = 0, 0.0, None
    for k in range(args.steps):
        ctx.submit_raw(pairs, MODE)
        if k > 0:
            last = ctx.complete()
            t = ctx.last_timing()
            launches += t["launches"]
            dp_ms += t["dp_ms"]
    last = ctx.complete()
    t = ctx.last_timing()
    launches += t["launches"]
    dp_ms += t["dp_ms"]
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    value, ms_max, cells_all = aggregate(cells * args.steps, ms, world)
    res = result_view(last).copy()
    fits = fit_all(res)
    parity = calibration_parity(txt, seqs, T, Ms, res, args.cal_len) if rank == 0 and args.parity_pairs > 0 else None

    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = n_sm * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = cells * args.steps * FLOPS_PER_CELL / (dp_ms / 1e3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": f"derived: {n_sm} SMs x 128 FP32 lanes x 2 x sm_max_mhz {sm_max:g} (of measured "
                               "clock; MEASURED_PEAKS.json has no FP32 figure)",
                "kernel": "dpKernel (mid), CUDA events on the library stream, per step",
                "algorithmic_flops_per_cell": FLOPS_PER_CELL}

    # e2e: each step copies the batch's sequences (2-bit packed) from host
    # memory, scores, copies the results back and fits every profile (FP64)
    words, mask, lens = d.pack_dna(seqs)
    ctx.clear_sequences()
    base = 0
    step_pairs = []
    for k in range(args.warmup + args.steps):
        step_pairs.append(pairs_for(list(range(base, base + len(seqs)))))
        base += len(seqs)
    for k in range(args.warmup):
        ctx.add_packed(words, lens, mask)
        ctx.score_pairs_raw(step_pairs[k], MODE)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(args.warmup, n_steps):
        ctx.add_packed(words, lens, mask)
        ctx.submit_raw(step_pairs[k], MODE)
        if k > args.warmup:
            fit_all(ctx.complete())
    fit_all(ctx.complete())
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    h2d = words.nbytes + mask.nbytes + 12 * len(lens) + 40 * len(seqs)
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": 40 * len(seqs), "note": "includes the FP64 fits of every profile on the host"}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_calibration_baseline(txt, seqs, T, args.cpu_seconds, args.seed)
    if rank == 0:
        print(json.dumps({
            "metric": "calibration batch fwd+bwd GCUPS (mid scores of every trial)", "value": value, "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args, world), cells_per_step=cells),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "parity": parity,
            "fits": {"lambda_median": float(np.median(fits[:, 0])), "K_median": float(np.median(fits[:, 1])),
                     "lambda_filter_median": float(np.median(fits[:, 2]))},
            "gpu_launches": launches, "clocks": clk, "dp_ms_per_step": dp_ms / args.steps,
            "launch": {"cuda_graph": not args.no_graph, "async_submit": True, "autotune": tuning}}), flush=True)
    ctx.close()


def run_reference(args, rank, world):
    if rank != 0:
        return
    if args.workload == "windows":
        genome, names, lens, pnames, plens, steps = windows_problem(args, 0)
        import dummest_b200 as d
        wins = d.windows_from_hits(steps[0], names, lens, pnames, plens)[0]
        vals, cb = [], None
        per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
        for _ in range(args.warmup + args.steps):
            cb = cpu_windows_baseline(genome, wins, names, per_step)
            vals.append(cb["value"])
        v = statistics.median(vals[args.warmup:]) if len(vals) > args.warmup else vals[-1]
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": "prefilter window stage: window nt decoded per second", "value": v,
            "unit": "Gnt/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic",
            "config": workload_config(args, world), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "Gnt/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    if args.workload == "calibration":
        profiles, txt, seqs = calibration_problem(args, 0)
        vals, cb = [], None
        per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
        for k in range(args.warmup + args.steps):
            cb = cpu_calibration_baseline(txt, seqs, args.cal_trials, per_step, args.seed + k)
            vals.append(cb["value"])
        v = statistics.median(vals[args.warmup:]) if len(vals) > args.warmup else vals[-1]
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": "calibration batch fwd+bwd GCUPS (mid scores of every trial)",
            "value": v, "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args, world), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    profiles, txt, steps = make_workload(args, 0, 1)
    if args.workload == "align":
        vals, cb = [], None
        per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
        for _ in range(args.warmup + args.steps):
            cb = cpu_align_baseline(txt, steps[0], args.al_gate, per_step)
            vals.append(cb["value"])
        v = statistics.median(vals[args.warmup:]) if len(vals) > args.warmup else vals[-1]
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": "hit-path traceback GCUPS (cells of every pair; hits traced)",
            "value": v, "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args, world), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    if args.workload == "search":
        import dummest_b200 as d
        rng = np.random.default_rng(args.seed)
        # gates from the library's calibration fits would need a GPU; the
        # reference arm calibrates with its own engine (estimateK, 200 x 3 kb)
        from oracle.ref import RefEngine
        e = RefEngine(32)
        e.set_rates()
        with tempfile.NamedTemporaryFile("w", suffix=".hmm", delete=False) as f:
            f.write(txt)
            path = f.name
        e.load_profiles(path)
        os.unlink(path)
        fits = []
        for p in range(len(profiles)):
            lam, k, lamf, kf = e.estimate_k(p, 3000, 100, 200, threads=os.cpu_count() or 1)
            fits.append({"lambda_filter": lamf, "K_filter": kf})
        gates = search_gates(fits, float(sum(len(r) for r in steps[0])))
        vals = []
        per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
        cb = None
        for _ in range(args.warmup + args.steps):
            cb = cpu_search_baseline(txt, steps[0], gates, per_step, int(rng.integers(1 << 30)))
            vals.append(cb["value"])
        v = statistics.median(vals[args.warmup:]) if len(vals) > args.warmup else vals[-1]
        cb["value"] = v
        print(json.dumps({
            "impl": "reference", "metric": "two-wave search GCUPS (cells of every pair)", "value": v,
            "unit": "GCUPS", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(args, world), "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}), flush=True)
        return
    vals = []
    cb = None
    per_step = max(args.cpu_seconds / max(args.steps, 1), 2.0)
    for _ in range(args.warmup + args.steps):
        cb = cpu_baseline(txt, steps[0], len(profiles), per_step, args.seed + len(vals))
        vals.append(cb["value"])
    v = statistics.median(vals[args.warmup:]) if len(vals) > args.warmup else vals[-1]
    cb["value"] = v
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GCUPS", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, world),
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "GCUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def genome_posterior_pass(ctx, sids, pid, windows, res, scan_ms):
    """The posterior pass of the genome scan: the windows whose mid score
    passes the hit gate minProbRatio = (K N / E)^(1/lambda) (dummest.cc:583-587,
    lambda and K from the profile's calibration, untimed; N the scanned
    length, E = 10) through dmst_posterior_summary (FP64 adjoint with the
    posterior tables reduced on the device), timed on its own."""
    import torch
    fit = ctx.estimate_k(pid, sequence_length=3000, border=100, trials=200)
    n_tot = float(sum(len(w) for w in windows))
    gate_ln = (np.log(fit["K"]) + np.log(n_tot) - np.log(SEARCH_E)) / fit["lambda"]
    above = np.nonzero(result_view(res)["mid_ln"] >= gate_ln)[0]
    if len(above) == 0:
        return {"windows_above": 0, "gate_bits": gate_ln / np.log(2.0)}
    M = ctx.profile_length(pid)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    logt, summ = ctx.posterior_summary([sids[k] for k in above], pid)
    wall = (time.perf_counter() - t0) * 1e3
    t = ctx.last_timing()
    cells = float(sum(len(windows[k]) for k in above)) * (M + 1)
    return {"windows_above": int(len(above)), "windows": len(windows), "gate_bits": gate_ln / np.log(2.0),
            "cells": cells, "wall_ms": wall, "adjoint_ms": t["dp_ms"], "null_ms": t["null_ms"],
            "gcups": cells / (wall / 1e3) / 1e9, "scan_plus_posterior_ms": scan_ms + wall,
            "output": "per window: column track of the largest cell posterior and its row, row sums of the match "
                      "posteriors (FP64; tables reduced on the device)"}


def run_ours(args, rank, world, local):
    import dummest_b200 as d
    from dummest_b200 import _ffi as F
    from dummest_b200 import shards
    import torch

    n_steps = args.warmup + args.steps
    profiles, txt, sets = make_workload(args, rank, n_steps, world)
    # Step k scores read set k mod len(sets): every set is distinct at one GPU
    # (20 timed steps of 5,000 reads are the configuration's 100,000 reads);
    # with N GPUs a step holds N times the reads, and the sets cycle.
    step_set = [k % len(sets) for k in range(n_steps)]
    # Batched pairs shard over the ranks (the cost-sorted pair queue, dealt
    # by strided interleaving; results gathered); the genome workload runs
    # one genome per rank.
    sharded = world > 1 and args.workload == "batched"
    dev = torch.device("cuda", local)
    ctx = d.Context(device=local, rows_per_lane=args.rows_per_lane)
    pids = ctx.load_hmm(txt)
    Ms = np.array([ctx.profile_length(p) for p in pids])

    def shares_of(recs):
        """Every rank's pair indices (profile-major pair order) and this rank's cells."""
        lens = np.array([len(r) for r in recs], np.int64)
        if not sharded:
            return [np.arange(len(lens) * len(pids))], float(lens.sum()) * float((Ms + 1).sum())
        costs = np.repeat(Ms + 1, len(lens)) * np.tile(lens, len(pids))
        shares = [shards.shard_indices(costs, world, r) for r in range(world)]
        return shares, float(costs[shares[rank]].sum())

    def rank_pairs(sids, shares):
        full = pair_array(sids, pids)
        if not sharded:
            return full
        mine = np.ascontiguousarray(full._keep[shares[rank]])
        out = (F.Pair * len(mine)).from_buffer(mine)
        out._keep = mine
        return out

    def finish(res, si):
        """A completed call's results: this rank's (one GPU), or every rank's
        gathered in pair order (NCCL all-gather through device memory)."""
        if not sharded:
            return res
        sh = set_shares[si]
        return shards.gather_results(result_view(res), sh[rank], n_pairs[si], sh, device=dev)

    # ---- value: reads resident in HBM ----
    set_sids, set_pairs, set_cells, set_shares, n_pairs = [], [], [], [], []
    for recs in sets:
        sids = ctx.add_dna(recs)
        shares, c = shares_of(recs)
        set_sids.append(sids)
        set_shares.append(shares)
        set_pairs.append(rank_pairs(sids, shares))
        set_cells.append(c)
        n_pairs.append(len(sids) * len(pids))
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    # Kernel shapes from the autotuner (untimed): every shape on the first
    # (warm-up) step's pairs, a sample large enough to fill the GPU.
    tuning = None
    if not args.no_autotune and args.rows_per_lane == 0:
        samp = set_sids[0][:2048]
        rates = ctx.autotune([s for _ in pids for s in samp], [p for p in pids for _ in samp])
        shapes = {}
        for M in Ms:
            key = "R%d/W%d" % ctx.tuned_shape(int(M))
            shapes[key] = shapes.get(key, 0) + 1
        short = ctx.tuned_rates("short")
        tuning = {"gcups_computed_cells": {f"R{r}/W{w}": round(v, 2) for (r, w), v in rates.items()},
                  "gcups_computed_cells_short_reads": {f"R{r}/W{w}": round(v, 2) for (r, w), v in short.items()},
                  "profiles_per_shape_long_reads": shapes, "sample_pairs": len(samp) * len(pids)}
    MODE = d.MODE_MID | (0 if args.no_graph else d.MODE_GRAPH)
    # Warm-up steps in the timed steps' pattern (each call submitted before the
    # previous one completes), so that both of the context's call slots hold
    # their buffers and launch graphs before the timed region.
    for w in range(args.warmup):
        if args.no_async:
            finish(ctx.score_pairs_raw(set_pairs[step_set[w]], MODE), step_set[w])
            continue
        ctx.submit_raw(set_pairs[step_set[w]], MODE)
        if w > 0:
            finish(ctx.complete(), step_set[w - 1])
    if args.warmup and not args.no_async:
        finish(ctx.complete(), step_set[args.warmup - 1])
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    # the timed calls' launches form the NVTX range "timed" (ncu --nvtx --nvtx-include timed/)
    torch.cuda.nvtx.range_push("timed")
    ev0.record(stream)
    launches, dp_ms, cells, exact_pairs = 0, 0.0, 0.0, 0
    kept = []  # (timed step, results) of every 4th timed step, for the parity sample
    parts = {"null_ms": 0.0, "dp_ms": 0.0, "exact_ms": 0.0, "host_ms": 0.0, "post_ms": 0.0, "wall_ms": 0.0}

    def account(res, k):
        t = ctx.last_timing()
        nonlocal launches, dp_ms, exact_pairs
        launches += t["launches"]
        dp_ms += t["dp_ms"]
        for key in parts:
            parts[key] += t[key]
        exact_pairs += int(np.count_nonzero(result_view(res)["flags"] & F.RES_EXACT_PATH))
        full = finish(res, step_set[k])
        if (k - args.warmup) % 4 == 0:
            kept.append((k, full))

    # Calls are submitted one ahead of their completion, so that the host work
    # of one step overlaps the device work of the previous one.
    for k in range(args.warmup, n_steps):
        if args.no_async:
            account(ctx.score_pairs_raw(set_pairs[step_set[k]], MODE), k)
        else:
            ctx.submit_raw(set_pairs[step_set[k]], MODE)
            if k > args.warmup:
                account(ctx.complete(), k - 1)
        cells += set_cells[step_set[k]]
    if not args.no_async:
        account(ctx.complete(), n_steps - 1)
    ev1.record(stream)
    torch.cuda.nvtx.range_pop()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    value, ms_max, cells_all = aggregate(cells, ms, world)
    exact_pairs = int(allreduce_sum(float(exact_pairs), world))
    # ---- parity of the timed results against the reference engine (after the timed region) ----
    parity = None
    if rank == 0 and args.parity_pairs > 0:
        parity = parity_sample(txt, [(sets[step_set[k]], r) for k, r in kept], args.parity_pairs, args.seed)
    posterior_pass = None
    if args.workload == "genome" and rank == 0:
        posterior_pass = genome_posterior_pass(ctx, set_sids[0], pids[0], sets[0], kept[-1][1], ms_max / args.steps)
    del kept

    # ---- roofline of the DP kernels (CUDA-event durations, this GPU) ----
    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = n_sm * 128 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s
    achieved = cells * FLOPS_PER_CELL / (dp_ms / 1e3) / 1e12
    tpc = traffic_per_cell()
    launch_cells = cells / args.steps
    roofline = {
        "bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s", "frac": achieved / fp32_peak,
        "traffic": (tpc * launch_cells) if tpc else None,
        "peak_source": f"derived: {n_sm} SMs x 128 FP32 lanes x 2 x sm_max_mhz {sm_max:g} (of measured clock; "
                       "MEASURED_PEAKS.json has no FP32 figure)",
        "kernel": "dpKernel (mid: backward + forward), CUDA events on the library stream, per step",
        "algorithmic_flops_per_cell": FLOPS_PER_CELL,
        "hbm_algorithmic_bytes_per_cell": 8,
        "hbm_frac_of_measured": (8 * cells / (dp_ms / 1e3)) / (peaks.get("hbm_gbs", 6451.2) * 1e9),
    }

    # ---- e2e: host buffers through the C ABI every step ----
    # Each step's reads are copied from host memory (2-bit packed) and decoded
    # on the device, scored, and the results copied back (and, with N GPUs,
    # gathered); steps are submitted one ahead of their completion.  The reads
    # of every step are appended (sequence ids continue), so the pair arrays
    # are built beforehand.
    packed = [d.pack_dna(recs) for recs in sets]
    ctx.clear_sequences()
    base = 0
    e2e_pairs = []
    for k in range(n_steps):
        si = step_set[k]
        e2e_pairs.append(rank_pairs(list(range(base, base + len(sets[si]))), set_shares[si]))
        base += len(sets[si])
    h2d = d2h = 0
    for w in range(args.warmup):  # in the timed steps' pattern, as above
        words, mask, lens = packed[step_set[w]]
        ctx.add_packed(words, lens, mask)
        if args.no_async:
            finish(ctx.score_pairs_raw(e2e_pairs[w], MODE), step_set[w])
            continue
        ctx.submit_raw(e2e_pairs[w], MODE)
        if w > 0:
            finish(ctx.complete(), step_set[w - 1])
    if args.warmup and not args.no_async:
        finish(ctx.complete(), step_set[args.warmup - 1])
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    next_id = sum(len(sets[step_set[w]]) for w in range(args.warmup))
    for k in range(args.warmup, n_steps):
        si = step_set[k]
        words, mask, lens = packed[si]
        sids = ctx.add_packed(words, lens, mask)
        assert sids[0] == next_id and len(sids) == len(lens)
        next_id += len(lens)
        pr = e2e_pairs[k]
        if args.no_async:
            finish(ctx.score_pairs_raw(pr, MODE), si)
        else:
            ctx.submit_raw(pr, MODE)
            if k > args.warmup:
                finish(ctx.complete(), step_set[k - 1])
        # packed reads + mask + offsets, then the per-pair descriptors the
        # library uploads (32 B pair + 8 B scratch offset) and the per-pair
        # results it reads back (16 B, and 24 B of exact-path results); with
        # N GPUs also this rank's results up for the all-gather and every
        # rank's results back down
        h2d += words.nbytes + mask.nbytes + 12 * len(lens) + 40 * len(pr)
        d2h += 40 * len(pr)
        if sharded:
            h2d += 40 * len(pr)
            d2h += 40 * n_pairs[si]
    if not args.no_async:
        finish(ctx.complete(), step_set[n_steps - 1])
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d // args.steps,
           "d2h_bytes_per_step": d2h // args.steps}
    if world > 1:
        e2e["bytes_note"] = "per rank"

    # ---- plain schedule on a sample of step pairs ----
    plain = None
    if rank == 0 and args.plain_pairs > 0:
        ctx.clear_sequences()
        recs = sets[step_set[args.warmup]]
        sids = ctx.add_dna(recs)
        rng = np.random.default_rng(args.seed)
        sel = rng.choice(len(sids) * len(pids), size=min(args.plain_pairs, len(sids) * len(pids)), replace=False)
        arr = (F.Pair * len(sel))()
        pc = 0.0
        for k, idx in enumerate(sel):
            p, s = pids[idx // len(sids)], sids[idx % len(sids)]
            arr[k].seq, arr[k].profile, arr[k].min_prob_ratio = s, p, -2.0
            pc += (Ms[p] + 1) * len(recs[idx % len(sids)])
        plain = {"pairs": len(sel), "cells": pc,
                 "kernel": "one pair per launch: one CTA of 8 warps sharing the pair's stripes (stripe pipeline, "
                           "fast-path arithmetic)",
                 "kernel_1warp": "one pair per launch: the batched kernel on a one-pair chunk (one warp computes)"}
        for key, flag in (("", d.MODE_PLAIN), ("_1warp", d.MODE_PLAIN | d.MODE_PLAIN_1WARP)):
            ctx.score_pairs_raw(arr, d.MODE_MID | flag)
            ctx.score_pairs_raw(arr, d.MODE_MID | flag)
            tp = ctx.last_timing()
            plain["gcups" + key] = pc / (tp["dp_ms"] / 1e3) / 1e9
            plain["launches" + key] = tp["launches"]
            plain["batched_over_plain" + key] = value / world / plain["gcups" + key]

    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_baseline(txt, sets[step_set[args.warmup]][:2 * args.reads_per_step], len(profiles),
                          args.cpu_seconds, args.seed)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "GCUPS", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args, world), cells_per_step=cells_all / args.steps,
                           distinct_read_sets=len(sets)),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "plain": plain, "parity": parity,
            **({"posterior_pass": posterior_pass} if posterior_pass else {}),
            "gpu_launches": launches, "exact_path_pairs": exact_pairs, "clocks": clk,
            "breakdown_ms_per_step": {k: v / args.steps for k, v in parts.items()},
            "launch": {"cuda_graph": not args.no_graph, "async_submit": not args.no_async, "autotune": tuning},
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def run_search(args, rank, world, local):
    import dummest_b200 as d
    from dummest_b200 import _ffi as F
    import torch

    n_steps = args.warmup + args.steps
    profiles, txt, steps = make_workload(args, rank, n_steps)
    ctx = d.Context(device=local)
    pids = ctx.load_hmm(txt)
    Ms = np.array([ctx.profile_length(p) for p in pids])

    def pairs_for(sids):
        return pair_array(sids, pids)

    # untimed: each profile's calibration (the filter wave's lambda and K) and
    # the kernel shapes
    fits = [ctx.estimate_k(p, 3000, 100, 200) for p in pids]
    step_sids = [ctx.add_dna(recs) for recs in steps]
    step_pairs = [pairs_for(sids) for sids in step_sids]
    gates = [search_gates(fits, float(sum(len(r) for r in recs))) for recs in steps]
    cells_step = [float(sum(len(r) for r in recs)) * float((Ms + 1).sum()) for recs in steps]
    samp = step_sids[0]
    ctx.autotune([s for _ in pids for s in samp], [p for p in pids for _ in samp])
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    for w in range(args.warmup):
        ctx.search_submit_raw(step_pairs[w], gates[w])
    while ctx.complete() is not None:
        pass
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    results, dp_ms, launches, cells = [], 0.0, 0, 0.0
    parts = {"null_ms": 0.0, "dp_ms": 0.0, "exact_ms": 0.0, "host_ms": 0.0}

    def account():
        nonlocal dp_ms, launches
        t = ctx.last_timing()
        dp_ms += t["dp_ms"]
        launches += t["launches"]
        for key in parts:
            parts[key] += t[key]
    for k in range(args.warmup, n_steps):
        ctx.search_submit_raw(step_pairs[k], gates[k])
        if k > args.warmup:
            results.append(ctx.complete())
            account()
        cells += cells_step[k]
    results.append(ctx.complete())
    account()
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    value, ms_max, cells_all = aggregate(cells, ms, world)
    # survivors' cells (the second wave's work)
    surv_cells = surv = 0
    for k, res in zip(range(args.warmup, n_steps), results):
        lens = np.array([len(r) for r in steps[k]], np.float64)
        for i, r in enumerate(res):
            if r.flags & F.RES_SURVIVOR:
                surv += 1
                surv_cells += (Ms[i // len(lens)] + 1) * lens[i % len(lens)]
    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    fp32_peak = n_sm * 128 * 2 * sm_max * 1e6 / 1e12
    achieved = (FILTER_FLOPS_PER_CELL * cells + FLOPS_PER_CELL * surv_cells) / (dp_ms / 1e3) / 1e12
    roofline = {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                "frac": achieved / fp32_peak, "traffic": None,
                "peak_source": f"derived: {n_sm} SMs x 128 FP32 lanes x 2 x sm_max_mhz {sm_max:g}",
                "kernel": "both waves' DP kernels and the survivor compaction, CUDA events on the library stream",
                "algorithmic_flops_per_cell": {"filter": FILTER_FLOPS_PER_CELL, "mid": FLOPS_PER_CELL}}
    # e2e: each step's reads copied (2-bit packed), decoded, searched, results copied back
    packed = [d.pack_dna(recs) for recs in steps]
    ctx.clear_sequences()
    base, e2e_pairs = 0, []
    for k in range(n_steps):
        e2e_pairs.append(pairs_for(list(range(base, base + len(steps[k])))))
        base += len(steps[k])
    for w in range(args.warmup):
        words, mask, lens = packed[w]
        ctx.add_packed(words, lens, mask)
        ctx.search_submit_raw(e2e_pairs[w], gates[w])
    while ctx.complete() is not None:
        pass
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for k in range(args.warmup, n_steps):
        words, mask, lens = packed[k]
        ctx.add_packed(words, lens, mask)
        ctx.search_submit_raw(e2e_pairs[k], gates[k])
        if k > args.warmup:
            ctx.complete()
        h2d += words.nbytes + mask.nbytes + 12 * len(lens) + 40 * len(e2e_pairs[k]) + 4 * len(pids)
        d2h += 57 * len(e2e_pairs[k])
    while ctx.complete() is not None:
        pass
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d // args.steps,
           "d2h_bytes_per_step": d2h // args.steps}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        cb = cpu_search_baseline(txt, steps[args.warmup], gates[args.warmup], args.cpu_seconds, args.seed)
    if rank == 0:
        print(json.dumps({
            "metric": "two-wave search GCUPS (cells of every pair)", "value": value, "unit": "GCUPS", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload_config(args, world), cells_per_step=cells / args.steps),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cb, "gpu_launches": launches, "clocks": clk,
            "survivors_per_step": surv / args.steps, "survivor_cell_fraction": surv_cells / cells,
            "breakdown_ms_per_step": {k: v / args.steps for k, v in parts.items()}}), flush=True)
    ctx.close()


def autograd_problem(args, rank):
    """The profile and one rank's reads."""
    from dummest_b200 import synth
    rng = np.random.default_rng(args.seed)
    prof = synth.make_profile(rng, args.ag_m, f"grad{args.ag_m}")
    rrng = np.random.default_rng(rank_seed(args.seed, rank))
    reads = synth.make_reads(rrng, args.ag_reads, args.ag_lmin, args.ag_lmax, [prof], 1.0, gc_range=(0.4, 0.6),
                             log_uniform=False)
    return prof, reads


def run_autograd(args, rank, world, local):
    import torch
    import dummest_b200 as d
    from dummest_b200 import autograd as ag
    from dummest_b200 import synth

    prof, reads = autograd_problem(args, rank)
    txt = synth.hmmer3_text([prof])
    _, values, params, bg = d.finalize_hmm(txt)
    M = args.ag_m
    ctx = d.Context(device=local)
    from dummest_b200 import _ffi as Fc
    ctx.adjoint_checkpoint({"on": Fc.ADJ_CKPT_ON, "off": Fc.ADJ_CKPT_OFF, "auto": Fc.ADJ_CKPT_AUTO}[args.ag_ckpt])
    sids = ctx.add_dna(reads)
    cells = float(sum(len(r) for r in reads)) * (M + 1)
    slot = ag.ProfileSlot(ctx, values, params, bg, sids)
    bg_row = torch.tensor(values[-1, 4:29], dtype=torch.float64)
    MI, MD, II, DD = synth.T_MI, synth.T_MD, synth.T_II, synth.T_DD
    em = torch.tensor(np.log(prof.match), requires_grad=True)
    tr = torch.tensor(np.tile(np.log([1 - MI - MD, MI, MD, 1 - II, II, 1 - DD, DD]), (M + 1, 1)),
                      requires_grad=True)
    fs = torch.tensor(np.log([0.0171, 0.0018, 0.0328, 0.0083]), requires_grad=True)
    opt = torch.optim.SGD([em, tr, fs], lr=1e-3)

    def step():
        opt.zero_grad()
        emit, par = ag.profile_params(em, tr, fs, bg_row)
        loss = -ag.log_likelihood(emit, par, slot) / len(reads)
        loss.backward()
        opt.step()
        return float(loss.detach())

    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local)
    for _ in range(args.warmup):
        step()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    adj_ms = null_ms = 0.0
    launches = 0
    losses = []
    for _ in range(args.steps):
        losses.append(step())
        t = ctx.last_timing()
        adj_ms += t["dp_ms"]
        null_ms += t["null_ms"]
        launches += t["launches"]
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    total_cells = cells * args.steps
    value, ms_max, cells_all = aggregate(total_cells, ms, world)
    peaks = measured_peaks()
    sm_max = peaks.get("sm_max_mhz", 1965.0)
    n_sm = torch.cuda.get_device_properties(local).multi_processor_count
    fp64_peak = n_sm * 64 * 2 * sm_max * 1e6 / 1e12  # TFLOP/s: 64 FP64 lanes per SM
    achieved = AG_FLOPS_PER_CELL * total_cells / (adj_ms / 1e3) / 1e12
    roofline = {
        "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
        "traffic": None,
        "peak_source": f"derived: {n_sm} SMs x 64 FP64 lanes x 2 x sm_max_mhz {sm_max:g} (of measured clock; "
                       "MEASURED_PEAKS.json has no FP64 figure)",
        "kernel": "adjointKernel (forward, then backward with the gradient sums), CUDA events on the library "
                  "stream, summed over the step's launches",
        "algorithmic_flops_per_cell": AG_FLOPS_PER_CELL,
        "adjoint_gcups": total_cells / (adj_ms / 1e3) / 1e9,
        "note": "latency-bound FP64 chains (a warp per pair, one row per lane): the fraction is low by design",
    }
    # e2e: the reads re-uploaded from host memory (2-bit packed) every step
    words, mask, lens = d.pack_dna(reads)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    h2d = d2h = 0
    for _ in range(args.steps):
        ctx.clear_sequences()
        slot.seq_ids = ctx.add_packed(words, lens, mask)
        step()
        # packed reads + mask + offsets, the per-pair descriptors and jobs, the
        # profile tables; back: log T per read and the gradient
        h2d += words.nbytes + mask.nbytes + 12 * len(lens) + 72 * len(lens) + 4 * (29 * (M + 1) + 11 * (M + 2))
        d2h += 8 * len(lens) + 8 * (11 * (M + 2) + 25 * (M + 1))
    torch.cuda.synchronize()
    e2e_s = allreduce_max(time.perf_counter() - t0, world)
    e2e = {"value": cells_all / e2e_s / 1e9, "unit": "GCUPS", "h2d_bytes_per_step": h2d // args.steps,
           "d2h_bytes_per_step": d2h // args.steps}
    cb = None
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import port
        v64, p64 = values.astype(np.float64), params.astype(np.float64)
        done_c, done_s, n = 0.0, 0.0, 0
        for r in reads:
            c = d.decode_dna(r)
            t = time.perf_counter()
            port.log_total(v64, p64, bg, c)
            done_s += time.perf_counter() - t
            done_c += (M + 1) * len(c)
            n += 1
            if done_s >= args.cpu_seconds:
                break
        cb = {"value": done_c / done_s / 1e9, "unit": "GCUPS", "cores": 1, "cpu_model": cpu_model(), "kind": "port",
              "sample": f"{n} reads of the step, {done_c:.3e} cells in {done_s:.1f} s: the oracle's FP64 log T "
                        "(one backward sweep, no gradient: the reference computes none), one core"}
    if rank == 0:
        line = {
            "metric": "log-likelihood + gradient GCUPS (adjoint, FP64)", "value": value, "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": dict(workload_config(args, world), cells_per_step=cells), "e2e": e2e, "roofline": roofline,
            "cpu_baseline": cb, "gpu_launches": launches, "clocks": clk,
            "breakdown_ms_per_step": {"null_ms": null_ms / args.steps, "adjoint_ms": adj_ms / args.steps},
            "loss_first_last": [losses[0], losses[-1]],
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def relaunch(n: int) -> int:
    """Runs this command again as n ranks, one process per GPU (torchrun on
    127.0.0.1); returns the launcher's exit status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # `bench.py --gpus N` outside a launcher: start the N ranks here
        sys.exit(relaunch(args.gpus))
    if args.impl == "reference" and args.workload == "autograd":
        rank, _, _ = dist_env()
        if rank == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the reference computes no gradient of its "
                              "likelihood (its search path scores only)"}), flush=True)
        return
    if args.impl == "reference":
        # The reference's CPU engine runs on rank 0 alone; it needs no process
        # group, and the other ranks exit without work.
        rank, world, _ = dist_env()
        if rank == 0:
            run_reference(args, rank, world)
        return
    rank, world, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        elif args.workload == "autograd":
            run_autograd(args, rank, world, local)
        elif args.workload == "search":
            run_search(args, rank, world, local)
        elif args.workload == "align":
            run_align(args, rank, world, local)
        elif args.workload == "windows":
            run_windows(args, rank, world, local)
        elif args.workload == "calibration":
            run_calibration(args, rank, world, local)
        else:
            run_ours(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
