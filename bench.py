#!/usr/bin/env python
"""Phases 1-4 of cf1-rs on B200: distinct k-mers classified per second.

Default workload: the 3.1 Gbp k=31 synthetic genome (workload 5: 25
chromosomes, ~50% repeats, poly-N every 10 Mb, 256 bins), generated seeded
in host memory (the reference's GRCh38 input is not available).  A step is
one pass of phases 1-4 over the whole genome: pack, minimizer histogram,
partition, super k-mer routing, per-bin sort + unique, MPHF construction and
classification into the 5-bit state vector.

  value : distinct k-mers / device time of a step, input resident in HBM
          (library CUDA events on its stream; the input is 3.1 GB, larger
          than the 126 MB L2, so steps do not reuse cached data)
  e2e   : the same metric through the C ABI from host buffers, one
          cf1gpu_run_streamed call per step: records in page-locked host
          memory DMA'd to the device in chunks while phase 1 scans, phases
          1-4, and the state words copied back into page-locked memory stage
          by stage while phase 4 runs; timed on the host around the call

With N GPUs (torchrun, one rank per GPU) the genome is sharded by bin, rank r
owning the bins b with b % N == r.  Default (--shard-mode exchange): every
rank scans only its 1/N of the genome in phase 1, the ranks all-reduce their
minimizer histograms (NCCL), route their super k-mer records to the bins'
owners in one NCCL all-to-all, and each runs phases 2-4 on what it received;
with --shard-mode replicated every rank routes the whole genome instead.
Either way the ranks all-gather their per-bin distinct counts (the global
slot offsets) inside each timed step; `value` is the genome's distinct
k-mers over the slowest rank's time (strong scaling).

Both MPHF forms run: plain per-bin GPU BBHash, and the learned index +
batched (persistent queue kernels) form; the headline is the faster one,
the other is reported beside it.  --impl reference times the CPU oracle port
(all host threads) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import re
import os
import statistics
import subprocess
import tempfile
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    1: dict(k=31, bins=128, name="1 record, 5 Mbp uniform ACGT, k=31"),
    2: dict(k=31, bins=128, name="transcriptome: 20k genes, 100k transcripts, k=31", short=True),
    3: dict(k=31, bins=128, name="repetitive genome 200 Mbp, 24 chromosomes, k=31"),
    4: dict(k=63, bins=128, name="repetitive genome 1 Gbp, 30 chromosomes, k=63"),
    5: dict(k=31, bins=256, name="human-scale synthetic genome 3.1 Gbp, 25 chromosomes, ~50% repeats, k=31"),
}
METRIC = "k-mers classified/s, 1 B200: learned-index vs GPU BBHash vs CPU (bit-exact)"
# What the CPU arm does: the oracle port's phase-3 semantics (canonical
# k-mers, radix sort, unique) and its classify.rs restatement over an exact
# rank map; it builds no minimizer histogram, no bins and no MPHF, so it does
# less than the reference's phases 1-4.
CPU_SCOPE = "oracle port: sort + unique + classify.rs restatement; no minimizer histogram, routing or MPHF"
UNIT = "distinct k-mers/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["gpu", "reference"], default="gpu")
    p.add_argument("--workload", type=int, default=5, choices=sorted(WORKLOADS))
    p.add_argument("--scale", type=float, default=1.0)
    p.add_argument("--forms", default="bbhash,learned")
    p.add_argument("--cpu-sample-mbp", type=float, default=40.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--leaf-size", type=int, default=0, help="learned index keys per leaf (0 = library default)")
    p.add_argument("--shard-mode", choices=["exchange", "replicated"], default="exchange",
                   help="N > 1: scan 1/N of the input per rank and swap records, or route it all on every rank")
    p.add_argument("--tuner-cache", default=os.path.join(tempfile.gettempdir(), "cf1_tuner_cache.txt"),
                   help="autotuner cache file (first warm-up run of an input class measures; '' = off)")
    p.add_argument("--state-update", choices=["phase3", "sideset", "cas"], default="phase3",
                   help="how the states are formed (library state_update): joined in the phase-3 dedup, or "
                        "classified per occurrence in phase 4 (side-set OR / CAS loop)")
    p.add_argument("--verify", choices=["auto", "on", "off"], default="auto",
                   help="after the timed steps, check every form's per-k-mer states on the whole workload against "
                        "the CPU oracle (auto: on with 1 GPU)")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def traffic_md(form: str, kernel: str) -> str:
    if kernel == "classify":
        return os.path.join(ROOT, "profiles", "classify_traffic_workload5_full.md")
    if form == "bbhash":
        return os.path.join(ROOT, "profiles", "wd_dedup_kernel_workload5_scale0.05.md")
    return os.path.join(ROOT, "profiles", "cs_sort_unique_kernel_workload5_scale0.05.md")


def committed_traffic(workload: int, scale: float, form: str, kernel: str = "classify"):
    """DRAM bytes (read + write) of one launch of the kernel, full size, from
    the committed ncu summary for the 3.1 Gbp workload (the summary says
    whether it was captured at full size or scaled from a smaller case); None
    for any other workload or scale, or when no summary exists."""
    if workload != 5 or scale != 1.0 or (kernel == "classify" and form != "bbhash"):
        return None
    try:
        with open(traffic_md(form, kernel)) as f:
            m = re.search(r"^traffic_bytes_per_launch = (\d+)$", f.read(), re.M)
        return int(m.group(1)) if m else None
    except OSError:
        return None


class Clocks:
    """nvidia-smi samples every 200 ms while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        self.t.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_sample(x, sample_bp: int):
    """First records of the workload up to sample_bp bases (a prefix of the
    first chromosome for genome workloads)."""
    off = x.offsets
    end = 0
    recs = [0]
    i = 0
    while i < len(off) - 1 and end < sample_bp:
        end = min(int(off[i + 1]), int(off[0]) + sample_bp)
        recs.append(end - int(off[0]))
        i += 1
    seq = np.ascontiguousarray(x.seq[int(off[0]):end])
    return seq, np.array(recs, dtype=np.uint64)


def run_cpu_baseline(x, k: int, sample_bp: int, threads: int):
    from oracle import oracle as o

    seq, off = cpu_sample(x, sample_bp)
    t0 = time.perf_counter()
    r = o.run(k, seq, off, nthreads=threads, method=0)
    dt = time.perf_counter() - t0
    return len(r.states) / dt, dt, len(seq), len(r.states)


def mem_available() -> int:
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) * 1024
    except OSError:
        pass
    return 16 << 30


def verify_forms(x, k: int, dumps: dict) -> dict:
    """Every form's (canonical k-mer, state) dump of the whole workload
    against the CPU oracle's classify.rs restatement, one hash partition of
    the k-mers at a time (as many partitions as host memory needs).  Runs
    after the timed region; the time it takes is reported, not timed."""
    from oracle import oracle as o

    threads = os.cpu_count() or 1
    w = 8 if k <= 32 else 16
    n_occ = max(1, len(x.seq))
    need = 3 * w * n_occ  # collected keys, their sort buffer and the per-block lists of one partition
    nparts = max(2, min(64, -(-need // max(1, int(0.4 * mem_available())))))
    log = lambda m: print(f"[verify] {m}", file=sys.stderr, flush=True)
    r = o.check_lists(k, x.seq, x.offsets, dumps, nparts=nparts, nthreads=threads, log=log)
    forms = r.pop("lists")
    r["oracle"] = "CPU restatement of src/classify.rs (method 0), keyed by canonical k-mer"
    r["forms"] = forms
    r["mismatches"] = sum(v["mismatches"] for v in forms.values())
    r["n_listed"] = {f: v["n_listed"] for f, v in forms.items()}
    return r


def reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import cf1_rs_b200 as cg

    wl = WORKLOADS[args.workload]
    x = cg.SynthInput(args.workload, scale=args.scale)
    threads = os.cpu_count() or 1
    sample_bp = int(args.cpu_sample_mbp * 1e6)
    for _ in range(args.warmup):
        run_cpu_baseline(x, wl["k"], sample_bp, threads)
    rates, secs = [], []
    for _ in range(args.steps):
        rate, dt, nb, nd = run_cpu_baseline(x, wl["k"], sample_bp, threads)
        rates.append(rate)
        secs.append(dt)
    value = len(rates) / sum(1.0 / r for r in rates)
    sample = f"first {nb / 1e6:.1f} Mbp of the workload ({nd} distinct k-mers) per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(secs),
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u64" if wl["k"] <= 32 else "u128",
        "data": "synthetic (seeded generator)",
        "config": {"workload": wl["name"], "k": wl["k"], "num_bins": wl["bins"], "scale": args.scale,
                   "parallelism": "cpu threads"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                         "scope": CPU_SCOPE},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU oracle port of phases 1-4 (phase-3 sort+dedup, classify.rs restatement); "
                "the Rust reference cannot be built here (no cargo)",
    }
    print(json.dumps(line), flush=True)


def gpu_arm(args):
    import torch
    import torch.distributed as dist

    import cf1_rs_b200 as cg
    from cf1_rs_b200 import sharded

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local))

    def maxall(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sumall(v: float) -> float:
        if world == 1:
            return v
        t = torch.tensor([v], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    def exchange_ms(g) -> float:
        """The shards' one exchange: all-gather of the per-bin distinct counts
        and the global slot offsets (device time on the current stream)."""
        if world == 1:
            return 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sharded.global_offsets(sharded.allgather_counts(g.bin_distinct_counts(), device="cuda"))
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    xchg = world > 1 and args.shard_mode == "exchange"

    def exchange_step(be) -> float:
        """One exchange-sharded step (scan, histogram all-reduce, routing,
        record all-to-all, phases 2-4, counts all-gather): device time on the
        current stream from before the scan to after the last collective."""
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        sharded.run_exchange(be, device="cuda", assemble=False)
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    wl = WORKLOADS[args.workload]
    k, bins = wl["k"], wl["bins"]
    verify = args.verify == "on" or (args.verify == "auto" and world == 1)
    if verify and world > 1:
        verify = False  # each rank holds its own bins only; the check runs on one GPU
    # strong scaling over bin shards: rank r keeps the bins b with
    # b % world == r (cf1_rs_b200.sharded)
    x = cg.SynthInput(args.workload, scale=args.scale, seed=0)
    # one cache file per rank (ranks run the same classes; no shared writes)
    tuner_path = (args.tuner_cache + (f".rank{rank}" if world > 1 else "")) if args.tuner_cache else None
    forms = {}
    clocks = Clocks(local)
    clock_info = None
    for form in args.forms.split(","):
        batched = form == "learned"
        copts = dict(mode=form, batched=batched, track_short_seqs=bool(wl.get("short")), tuner_cache=tuner_path,
                     learned_leaf_size=args.leaf_size, state_update=args.state_update)
        be = sharded.GpuExchangeBackend(k, bins, rank, world, device=local, **copts) if xchg else None
        g = be.ctx if xchg else cg.Cf1Gpu(k=k, num_bins=bins, device=local, shard_index=rank, shard_count=world,
                                          **copts)
        g.add_records(x.seq, x.offsets)
        g.upload()

        def step() -> float:
            if xchg:
                return exchange_step(be)
            g.run_resident()
            return g.stats()["ms_total"] + exchange_ms(g)

        for _ in range(args.warmup):
            step()
        barrier()
        if clock_info is None:
            clocks.start()
        ms, ms_cls, ms_dd, launches, phase = [], [], [], 0, {}
        for _ in range(args.steps):
            ms.append(step())
            s = g.stats()
            ms_cls.append(s["ms_classify_kernel"])
            ms_dd.append(s["ms_dedup_kernel"])
            launches += s["n_kernel_launches"]
            for key in ("ms_phase1", "ms_phase2", "ms_phase3_sort", "ms_phase3_mphf", "ms_phase4"):
                phase[key] = phase.get(key, 0.0) + s[key] / args.steps
        barrier()
        if clock_info is None:
            clock_info = clocks.stop()
        # after the timed steps (untimed): the form's (key, state) list for the
        # oracle check, if host memory holds it beside the check's own needs
        dump = None
        if verify:
            w_key = 8 if k <= 32 else 16
            n_d = int(s["n_distinct"])
            held = sum(v["dump"][0].nbytes + v["dump"][1].nbytes for v in forms.values() if v.get("dump"))
            need = n_d * (w_key + 2) + len(x.seq) + 3 * w_key * len(x.seq) // 16 + (8 << 30)
            if mem_available() > need:
                dump = g.dump_states()
            else:
                print(f"[verify] {form}: not checked, host memory ({mem_available() >> 30} GiB free, "
                      f"{held >> 30} GiB held) is short of {need >> 30} GiB", file=sys.stderr, flush=True)
        total_ms = maxall(sum(ms))
        distinct = sumall(s["n_distinct"])
        forms[form] = dict(
            value=distinct * args.steps / (total_ms / 1e3), ms_per_step=total_ms / args.steps,
            ms_classify_kernel=maxall(statistics.mean(ms_cls)), ms_dedup_kernel=maxall(statistics.mean(ms_dd)),
            launches=launches, stats=s,
            phases_ms={k2: round(v, 3) for k2, v in phase.items()},
            learned=g.learned_stats() if form == "learned" else None, ctx=g, be=be, dump=dump,
            image_bytes=g.mphf_image_bytes())
        if form != args.forms.split(",")[-1]:
            g.close()
            forms[form]["ctx"] = None
    head_name = max(forms, key=lambda f: forms[f]["value"])
    head = forms[head_name]
    s = head["stats"]
    for f in forms.values():  # one context at a time on the device
        if f is not head and f["ctx"] is not None:
            f["ctx"].close()
            f["ctx"] = None
    # ---- end to end through the C ABI from host buffers
    e2e = None
    if not args.no_e2e:
        g, be = head["ctx"], head["be"]
        if g is None:
            copts = dict(mode=head_name, batched=head_name == "learned", track_short_seqs=bool(wl.get("short")),
                         tuner_cache=tuner_path, learned_leaf_size=args.leaf_size, state_update=args.state_update)
            be = sharded.GpuExchangeBackend(k, bins, rank, world, device=local, **copts) if xchg else None
            g = be.ctx if xchg else cg.Cf1Gpu(k=k, num_bins=bins, device=local, shard_index=rank,
                                              shard_count=world, **copts)
        # inputs and the result in page-locked host memory: the records go to
        # the device in one DMA, the state words come back in one
        pin_seq = torch.empty(max(1, x.seq.nbytes), dtype=torch.uint8, pin_memory=True)
        seq_h = pin_seq.numpy()[: x.seq.nbytes]
        seq_h[:] = x.seq
        nw = (s["n_distinct"] + 11) // 12
        pin_words = torch.empty(max(1, 8 * nw), dtype=torch.uint8, pin_memory=True)
        words = pin_words.numpy()[: 8 * nw].view(np.uint64)
        times = []
        for i in range(args.warmup + args.steps):
            barrier()
            t0 = time.perf_counter()
            if xchg:  # page-locked records DMA'd in, the shard's words copied back
                g.reset_input()
                g.add_records(seq_h, x.offsets)
                sharded.run_exchange(be, device="cuda", assemble=False)
                g.states(words[: (g.total_kmers() + 11) // 12])
            else:
                g.run_streamed(seq_h, x.offsets, words)  # copies overlapped with phases 1 and 4
                exchange_ms(g)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                times.append(dt)
        e2e_s = maxall(sum(times))
        e2e = {"value": sumall(s["n_distinct"]) * args.steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": int(sumall(s["n_bases"] + s["n_records"])),
               "d2h_bytes_per_step": int(sumall(words.nbytes)), "ms_per_step": 1e3 * e2e_s / args.steps}
        g.close()
    for f in forms.values():
        if f["ctx"] is not None:
            f["ctx"].close()
        f["ctx"] = None
    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    peaks, peak_kind = measured_peaks()
    L = s["n_bases"] + s["n_records"]
    n_occ, n_dist = s["n_kmer_occurrences"], s["n_distinct"]
    w = 8 if k <= 32 else 16
    # classification per occurrence (state_path 1, 2): 2-bit sequence read
    # once + one 32-B sector read and one written per occurrence (state word
    # RMW); MPHF probes excluded
    b4 = 0.25 * L + 64.0 * n_occ
    if int(s["state_path"]) == 0:
        # states joined in phase 3: the dominant kernel is the shared-memory
        # dedup, which reads every occurrence's key and side-set byte and
        # writes every distinct key and its joined byte (+ in the BBHash form
        # BBHash level 0: 8 bits per occurrence, stored as 16-B {bits, rank}
        # entries per 64 bits, i.e. 2 B per occurrence)
        # The BBHash form with 64-bit keys and a split of >= 6 bits runs the
        # multisplit on packed words (the byte inside the key's word), so the
        # dedup reads w bytes per occurrence there
        packed = head_name == "bbhash" and w == 8 and 6 <= int(s["sort_msd_bits"]) <= 64
        b_dd = (w if packed else w + 1.0) * n_occ + (w + 1.0) * n_dist + (2.0 * n_occ if head_name == "bbhash" else 0.0)
        ach = b_dd / (head["ms_dedup_kernel"] / 1e3) / 1e9
        # BBHash form: the warp dedup, with the block kernel for the few
        # sub-buckets it leaves (timed together); learned form: the sorted
        # chunk dedup
        kname = "wd_dedup_kernel" if head_name == "bbhash" else "cs_sort_unique_kernel"
        roofline = {"kernel": kname, "bound": "hbm", "achieved": ach, "peak": peaks["hbm_gbs"],
                    "unit": "GB/s", "frac": ach / peaks["hbm_gbs"], "peak_kind": peak_kind,
                    "traffic": committed_traffic(args.workload, args.scale, head_name, "dedup"),
                    "algorithmic_bytes": b_dd}
    else:
        ach = b4 / (head["ms_classify_kernel"] / 1e3) / 1e9
        roofline = {"kernel": "classify_defer_kernel" if head_name == "bbhash" else "classify_kernel", "bound": "hbm",
                    "achieved": ach, "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": ach / peaks["hbm_gbs"],
                    "peak_kind": peak_kind, "traffic": committed_traffic(args.workload, args.scale, head_name),
                    "algorithmic_bytes": b4}
    # whole phases 1-4: input read once, records written + read, keys
    # written + read by the sort, distinct keys written and read by the MPHF
    # build, plus the classification bytes above
    s_bins = 8.0 * s["n_superkmers"]
    b14 = 0.25 * L + 2 * s_bins + 2 * w * n_occ + 2 * w * n_dist + b4
    pipe = {"achieved": b14 / (head["ms_per_step"] / 1e3) / 1e9, "unit": "GB/s", "algorithmic_bytes": b14,
            "frac": b14 / (head["ms_per_step"] / 1e3) / 1e9 / peaks["hbm_gbs"]}
    parity = None
    if verify:
        dumps = {f: v.pop("dump") for f, v in forms.items() if v.get("dump") is not None}
        parity = verify_forms(x, k, dumps) if dumps else {"checked": False, "why": "host memory"}
        del dumps
    cpu = None
    if not args.no_cpu_baseline:
        rate, dt, nb, nd = run_cpu_baseline(x, k, int(args.cpu_sample_mbp * 1e6), os.cpu_count() or 1)
        cpu = {"value": rate, "unit": UNIT, "cores": os.cpu_count() or 1, "kind": "port",
               "sample": f"first {nb / 1e6:.1f} Mbp of the workload ({nd} distinct k-mers), {dt:.1f} s",
               "scope": CPU_SCOPE}
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "u64" if k <= 32 else "u128", "data": "synthetic (seeded generator)",
        "config": {"workload": wl["name"], "k": k, "num_bins": bins, "scale": args.scale, "form": head_name,
                   "bases": int(s["n_bases"]), "records": int(s["n_records"]), "distinct_kmers": int(n_dist),
                   "kmer_occurrences": int(n_occ),
                   "parallelism": f"bin shards x{world} ({args.shard_mode})" if world > 1 else "1 GPU",
                   "l2": "input 3.1 GB > 126 MB L2 (no flush needed)"},
        "bp_per_s": s["n_bases"] / (head["ms_per_step"] / 1e3),
        "roofline": roofline,
        "roofline_phases_1_4": pipe,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "clocks": clock_info,
        "parity": parity if parity is not None else {"checked": False},
        "gpu_launches": int(head["launches"]),
        "forms": {f: {"value": v["value"], "ms_per_step": v["ms_per_step"],
                      "ms_classify_kernel": v["ms_classify_kernel"], "phases_ms": v["phases_ms"],
                      "bbhash_levels": int(v["stats"]["bbhash_levels"]), "mphf_bytes": int(v["stats"]["mphf_bytes"]),
                      "mphf_image_bytes": int(v["image_bytes"]), "state_path": int(v["stats"]["state_path"]),
                      "dedup_overflow": int(v["stats"]["dedup_overflow"]),
                      "ms_dedup_kernel": v["ms_dedup_kernel"],
                      "sort": ("lsd" if v["stats"]["sort_msd_bits"] == 2**64 - 1
                               else f"msd{v['stats']['sort_msd_bits']}"),
                      "learned_bins": int(v["stats"]["learned_bins"]), "fallback_bins": int(v["stats"]["fallback_bins"]),
                      "sk_tile": int(v["stats"]["sk_tile"]),
                      "tuner": ["off", "cache", "measured"][int(v["stats"]["tuner_state"])],
                      "learned": v["learned"]} for f, v in forms.items()},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
