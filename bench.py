#!/usr/bin/env python
"""Benchmark of the B200 MSD radix string sort (one JSON line on rank 0).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload urls_50m|zipf_words_100m|uniform_1m|batch_c4|serve_c5|
                              text_urls_50m|suffixes_160m]

A step is one complete sort of the workload (perm + LCP) from inputs resident
in HBM.  `value` is strings/s over the whole job; `e2e` repeats the
measurement through the host-buffer entry point (ssort_sort_host) with the
host<->device copies inside the timed region.  The plain sort is a
single-GPU routine: with N GPUs every rank sorts its own replica of the
workload ("replicas", weak scaling) and the time is the max over ranks.

--impl reference times the reference's own msd_CE6 (compiled from its sources
into oracle/_ref/libref.so) on the host cores, on a bounded sample of the same
workload per step.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "string-sorting_b200"))

import numpy as np  # noqa: E402

import pyssort  # noqa: E402

METRIC = "sort throughput (strings/s)"
PARAMS = {"target_bucket": pyssort.SSORT_PARAM_TARGET_BUCKET,
          "warp8_cap": pyssort.SSORT_PARAM_WARP8_CAP,
          "overlap": pyssort.SSORT_PARAM_OVERLAP,
          "fused_gather": pyssort.SSORT_PARAM_FUSED_GATHER,
          "warp1_deep": pyssort.SSORT_PARAM_WARP1_DEEP,
          "block_prefetch": pyssort.SSORT_PARAM_BLOCK_PREFETCH,
          "graph": pyssort.SSORT_PARAM_GRAPH,
          "l2_prefetch": pyssort.SSORT_PARAM_L2_PREFETCH,
          "digit_bits": pyssort.SSORT_PARAM_DIGIT_BITS,
          "scatter": pyssort.SSORT_PARAM_SCATTER,
          "block_lean": pyssort.SSORT_PARAM_BLOCK_LEAN,
          "match_vote": pyssort.SSORT_PARAM_MATCH_VOTE,
          "warp_merge": pyssort.SSORT_PARAM_WARP_MERGE,
          "scan": pyssort.SSORT_PARAM_SCAN}


def apply_params(sorter, args):
    """--param NAME=VALUE settings (and the older dedicated flags)."""
    out = {}
    for kv in getattr(args, "param", []) or []:
        k, v = kv.split("=", 1)
        sorter.set_param(PARAMS[k], int(v))
        out[k] = int(v)
    if getattr(args, "target_bucket", 0):
        sorter.set_param(pyssort.SSORT_PARAM_TARGET_BUCKET, args.target_bucket)
        out["target_bucket"] = args.target_bucket
    if getattr(args, "warp1_deep", None) is not None:
        sorter.set_param(pyssort.SSORT_PARAM_WARP1_DEEP, args.warp1_deep)
        out["warp1_deep"] = args.warp1_deep
    return out
# Wall-clock bound of the reference arm's timed steps (seconds): a full-size
# CPU sort of the 50 M URLs takes about 14 s on one core.
REF_BUDGET_S = 300.0
# Most distinct requests one serving sweep generates up front (about 17 MB of
# keys each on average, held in pinned host memory and in HBM).
SERVE_FRESH_CAP = 1200
UNIT = "strings/s"
DEFAULT_WORKLOAD = "urls_50m"
CPU_SAMPLE = {"urls_50m": 4_000_000, "zipf_words_100m": 8_000_000, "uniform_1m": 1_000_000,
              "text_urls_50m": 4_000_000, "suffixes_160m": 16_000_000}
DESCRIPTIONS = {
    "urls_50m": "50,000,000 URLs: 'http://' + Zipf(1.1) host of 4,096 (8-24 [a-z]) + 1-6 "
                "'/'-segments of 3-12 [a-z0-9]; seed 2; uint64 offsets",
    "zipf_words_100m": "100,000,000 copies of Zipf(1.0) words from 1,000,000 distinct "
                       "geometric(0.15)-length [a-z] words clipped to [1,24]; seed 3; uint64 offsets",
    "uniform_1m": "1,000,000 strings, length U[1,20], bytes U{'a'..'z'}; seed 1",
    "batch_c4": "independent instances, counts log-uniform in [100, 2,000,000], alphabet "
                "{4 from 'A', 26 from 'a', 95 from ' '}, length U[1, L], L in {8, 32, 128}; "
                "the instance list stops at 1.5e9 expected key bytes; seeds 5 (list), 4 (strings)",
    "text_urls_50m": "the urls_50m strings as one text file: resident steps find the starts of "
                     "the NUL-delimited (--raw) text on the GPU, then sort; e2e sorts the "
                     "'\\n'-delimited file (default mode) from pinned host memory; uint32 offsets",
    "suffixes_160m": "every suffix (--suffix-sorting) of a 160,000,000-byte text: Zipf(1.0) "
                     "words (as zipf_words_100m, seed 8) separated by spaces, overwritten by "
                     "2,000 copies of earlier passages of log-uniform length in [32, 4096] "
                     "bytes; uint32 offsets",
    "serve_c5": "Poisson request stream swept over 1k-50k req/s; request string counts "
                "log-uniform in [1,000, 5,000,000], strings as batch_c4; every request a "
                "distinct, freshly generated one (generated before the sweep, in pinned host "
                "memory); uint32 offsets; 120 GB arena budget",
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD,
                    choices=sorted(pyssort.WORKLOADS) + ["batch_c4", "batch_c4_full", "serve_c5",
                                                         "text_urls_50m", "suffixes_160m"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--autotune", action="store_true",
                    help="run ssort_autotune on the input before timing (reported in `tuning`)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the other configurations measured beside the default one")
    ap.add_argument("--warp1-deep", type=int, default=None,
                    help="in-warp refinement steps of the one-per-lane sort (library default "
                         "when absent)")
    ap.add_argument("--target-bucket", type=int, default=0,
                    help="override the partition's wanted strings per range bucket")
    ap.add_argument("--param", action="append", default=[], metavar="NAME=VALUE",
                    help="set a tuning parameter of the sort context (names: " +
                         ", ".join(sorted(PARAMS)) + "); repeatable")
    ap.add_argument("--serve-requests", type=int, default=300,
                    help="requests per arrival rate of the serve_c5 sweep")
    ap.add_argument("--serve-rates", default="1000,5000,20000,50000")
    ap.add_argument("--serve-pool", type=int, default=64,
                    help="distinct requests the serve_c5 stream draws from (without --serve-fresh)")
    ap.add_argument("--serve-pooled", dest="serve_fresh", action="store_false",
                    help="draw the sweep's requests from a pool of --serve-pool distinct "
                         "requests instead of generating every request afresh")
    ap.add_argument("--serve-budget-gb", type=float, default=120.0)
    ap.add_argument("--serve-max-strings", type=int, default=1 << 27)
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the workload's string count (profiling runs only; "
                         "the reported workload is the full one at 1.0)")
    return ap.parse_args()


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ---- clocks sampler -----------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.gpu)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                self.rows.append(parts)

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        sm = [num(r[1]) for r in self.rows if num(r[1]) is not None]
        mx = [num(r[2]) for r in self.rows if num(r[2]) is not None]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ---- algorithmic bytes -----------------------------------------------------------
KB = 16  # key bytes per round

# DRAM bytes (read + write) per string handled, from one ncu capture of every
# launch of three sorts of 10 M URLs (dram__bytes_read/write summed per kernel
# and divided by the strings the kernel handled); scaled by the strings a
# launch handles to give `roofline.traffic` per launch.  Writes that stay in
# L2 until a later kernel evicts them are not counted here.
TRAFFIC_WORKLOAD = "urls_50m"
TRAFFIC_PER_STRING = {
    "count_gather": 120.3,  # round 1 from the kept copies, round 2 random offset + key reads
    "gather": 95.0,         # round 0: the arena streamed in order, bytes 16..31 kept
    "count": 17.9,
    "scatter": 36.3,
    "block": 57.2,
    "warp8": 195.0,
    "warp1": 261.0,
}


def kernel_strings(st):
    """Strings each kernel handled during one sort (stats counters)."""
    return {
        "gather": st.gather_elems - st.gather_fused,
        "count_gather": st.gather_fused, "count": st.partitioned - st.gather_fused,
        "scatter": st.partitioned,
        "warp1": st.warp1_fresh + st.warp1_keyed, "warp8": st.warp8_fresh + st.warp8_keyed,
        "block": st.block_fresh + st.block_keyed,
    }


def kernel_bytes(st, w):
    """Algorithmic bytes each kernel must move for one sort, from the per-kernel
    string counts: the first partition level of a round gathers while it
    counts: it reads idx (4) + offset (w) + the key bytes and writes the key
    (16); later levels' count reads keys (16); scatter reads and writes key+idx
    (2x20); on-chip sorts read idx (4) + offset (w) + key bytes when they
    gather themselves, or key+idx (20) otherwise, and write idx + lcp (8);
    equality buckets copy idx (8) and/or write lcp (4)."""
    def sort_bytes(fresh, keyed):
        return fresh * (4 + w + KB) + keyed * (KB + 4) + (fresh + keyed) * 8
    # Round 0's gather may also keep key bytes 16..31 per string (read 16 more,
    # write 16); round 1's first level then reads those (idx 4 + 16) instead of
    # the offset and the arena, in whichever kernel gathers that level.  Round
    # 0 gathers in a separate pass whenever any round does (a small round 0
    # gathers inside its count, and so does every round under mode 2).
    saved = getattr(st, "window_saved", 0)
    used = getattr(st, "window_used", 0)
    used_by = "count_gather" if st.gather_fused else "gather"
    saved_by = "gather" if st.gather_elems > st.gather_fused else "count_gather"
    out = {
        "gather": (st.gather_elems - st.gather_fused) * (4 + w + KB + KB),
        "count_gather": st.gather_fused * (4 + w + KB + KB),
        "count": (st.partitioned - st.gather_fused) * KB,
        "scatter": st.partitioned * 2 * (KB + 4),
        "warp1": sort_bytes(st.warp1_fresh, st.warp1_keyed),
        "warp8": sort_bytes(st.warp8_fresh, st.warp8_keyed),
        "block": sort_bytes(st.block_fresh, st.block_keyed),
        "equal": st.equal_moved * 8 + st.equal_final * 4,
    }
    out[saved_by] += saved * 2 * KB
    out[used_by] -= used * w
    return out


def intrinsic_live(lcp, n):
    """Strings live entering each 8-byte round of a plain MSD radix sort,
    derived from the final LCP array (independent of this implementation's
    round width): string i is live at depth 8r when it shares >= 8r bytes
    with a neighbour, i.e. max(lcp[i], lcp[i+1]) >= 8r."""
    import numpy as np
    l = np.asarray(lcp, dtype=np.int64)
    m = np.maximum(l, np.append(l[1:], 0))
    if not n:
        return [0]
    # m >= 8r exactly when m // 8 >= r: one histogram, then suffix sums
    ge = np.cumsum(np.bincount(m // 8)[::-1])[::-1]
    return [n] + [int(x) for x in ge[1:]]


def sort_algorithmic_bytes(live8, n, w):
    """Bytes a plain 8-byte-per-round MSD radix sort must touch: per live
    string per round idx (4) + offset (w) + 8 key bytes + one read and one
    write of (key, idx) (2x12); plus the perm and lcp writes (8 per string)."""
    return sum(m * (4 + w + 8 + 24) for m in live8) + n * 8


# ---- our arm ---------------------------------------------------------------------
def max_over_ranks(dist, x, device):
    """The largest of every rank's x (every rank calls this with its own);
    x itself without a process group."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank, steps, world, seconds):
    """Whole-job throughput of replicas: every rank processed units_per_rank
    per step, and the job took the slowest rank's time."""
    return units_per_rank * steps * world / seconds


def run_ours(args, rank, world, local_rank, dist):
    import torch
    torch.cuda.set_device(local_rank)
    ss = pyssort.WORKLOADS[args.workload](args.scale)
    n = ss.n
    w = ss.offs.dtype.itemsize
    arena_t = torch.from_numpy(ss.arena)
    d_arena = arena_t.to(f"cuda:{local_rank}")
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).to(f"cuda:{local_rank}")
    d_perm = torch.empty(n, dtype=torch.int32, device=f"cuda:{local_rank}")
    d_lcp = torch.empty(n, dtype=torch.int32, device=f"cuda:{local_rank}")
    sorter = pyssort.Sorter(local_rank)
    params = apply_params(sorter, args)
    stream = torch.cuda.Stream(device=local_rank)
    ab = ss.arena.nbytes

    def step():
        sorter.sort_device(d_arena, ab, d_offs, w, n, d_perm, d_lcp, stream=stream.cuda_stream)

    tuning = sorter.autotune(d_arena, ab, d_offs, w, n) if args.autotune else None

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    clocks = Clocks(local_rank)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        dist.barrier()
    # Per-kernel times from a second pass with an event pair around every
    # launch; profiling runs every kernel on the sort's stream, one after the
    # other (the timed pass above overlaps the on-chip sorts with the
    # partition levels), so these are the kernels' own durations.
    sorter.set_profiling(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    ktimes = sorter.kernel_times()
    sorter.set_profiling(False)
    st = sorter.stats()

    ms = max_over_ranks(dist, ms, f"cuda:{local_rank}")

    # ---- end to end through the host-buffer entry point (pinned buffers) ------
    e2e = None
    if not args.no_e2e:
        h_arena = torch.empty(ab, dtype=torch.uint8, pin_memory=True)
        h_arena.numpy()[:] = ss.arena
        h_offs = torch.empty(n, dtype=torch.int64, pin_memory=True)
        h_offs.numpy()[:] = ss.offs.view(np.int64)
        h_perm = torch.empty(n, dtype=torch.int32, pin_memory=True)
        h_lcp = torch.empty(n, dtype=torch.int32, pin_memory=True)
        na, no = h_arena.numpy(), h_offs.numpy().view(np.uint64)
        pp, pl = h_perm.numpy().view(np.uint32), h_lcp.numpy().view(np.uint32)
        sorter.sort_host(na, no, perm=pp, lcp=pl)  # warm the staging buffers

        def timed_host(lcp_out):
            if dist is not None:
                dist.barrier()
            t0 = time.perf_counter()
            for _ in range(args.steps):
                sorter.sort_host(na, no, with_lcp=lcp_out is not None, perm=pp, lcp=lcp_out)
            return max_over_ranks(dist, time.perf_counter() - t0, f"cuda:{local_rank}")

        # The reference routine returns the order only, so the headline reads
        # back the permutation; the same call with the LCP array is beside it.
        e2e_s = timed_host(None)
        e2e_lcp_s = timed_host(pl)
        # The caller hands over 8-byte offsets; ssort_sort_host narrows them
        # to 4 bytes on the host (during the arena copy) when the arena is
        # below 4 GB and n >= 2^20, so that is what crosses the link.
        link_w = 4 if (ab + 16 <= 0xFFFFFFFF and n >= (1 << 20)) else 8
        e2e = {"value": job_rate(n, args.steps, world, e2e_s), "unit": UNIT,
               "h2d_bytes_per_step": int(ab + n * link_w), "d2h_bytes_per_step": int(n * 4),
               "caller_bytes_per_step": int(ab + n * 8),
               "ms_per_step": 1000 * e2e_s / args.steps,
               "api": "ssort_sort_host (pinned host buffers, 8-byte offsets), permutation read back",
               "with_lcp": {"value": job_rate(n, args.steps, world, e2e_lcp_s),
                            "d2h_bytes_per_step": int(n * 8),
                            "ms_per_step": 1000 * e2e_lcp_s / args.steps}}
        del h_arena, h_offs, h_perm, h_lcp
        dropin = time_dropin(ss, n, max(1, min(args.steps, 5))) if world == 1 else None
        if dropin is not None:
            e2e["dropin"] = dropin
    clocks.stop()

    if rank != 0:
        return None

    # ---- roofline of the dominant kernel ---------------------------------------
    peak, peak_kind = peaks()
    kb = kernel_bytes(st, w)
    per_kernel = {}
    for name, (kms, launches) in ktimes.items():
        entry = {"ms_total": round(kms, 4), "launches": int(launches),
                 "ms_per_step": round(kms / args.steps, 4)}
        if name in kb:
            entry["algorithmic_bytes_per_step"] = int(kb[name])
            entry["gbs"] = round(kb[name] * args.steps / (kms / 1e3) / 1e9, 1) if kms > 0 else None
        per_kernel[name] = entry
    timed = {k: v for k, v in per_kernel.items() if k in kb}
    dom = max(timed, key=lambda k: timed[k]["ms_total"]) if timed else None
    roofline = None
    if dom:
        d = per_kernel[dom]
        per_launch_bytes = kb[dom] * args.steps / d["launches"]
        per_launch_s = d["ms_total"] / 1e3 / d["launches"]
        ach = per_launch_bytes / per_launch_s / 1e9
        traffic = None
        # measured DRAM bytes exist only for the URL workload's kernels
        if dom in TRAFFIC_PER_STRING and args.workload == TRAFFIC_WORKLOAD:
            strings_per_launch = kernel_strings(st)[dom] * args.steps / d["launches"]
            traffic = int(TRAFFIC_PER_STRING[dom] * strings_per_launch)
        roofline = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 4),
                    "traffic": traffic, "algorithmic_bytes_per_launch": int(per_launch_bytes),
                    "launch_ms": round(per_launch_s * 1e3, 4)}
    live8 = intrinsic_live(d_lcp.cpu().numpy().view(np.uint32), n)
    sort_bytes = sort_algorithmic_bytes(live8, n, w)
    sort_s = ms / 1e3 / args.steps
    sort_roof = {"bound": "hbm", "algorithmic_bytes_per_sort": int(sort_bytes),
                 "achieved": round(sort_bytes / sort_s / 1e9, 1), "peak": peak,
                 "frac": round(sort_bytes / sort_s / 1e9 / peak, 4),
                 "frac_of_8tbs": round(sort_bytes / sort_s / 1e9 / 8000, 4),
                 "live_per_8byte_round": live8,
                 "formula": "sum_r m_r*(4+W+8+24) + n*8, m_r from the LCP array"}
    launches = sum(v["launches"] * (3 if k == "scan" else 1) for k, v in per_kernel.items())

    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(args.workload, ss)

    lens_mean = ss.text_bytes / n - 1
    out = {
        "metric": METRIC, "value": job_rate(n, args.steps, world, ms / 1e3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": args.workload, "description": DESCRIPTIONS.get(args.workload),
                   "n_strings": n, "key_bytes": int(ss.text_bytes), "mean_len": round(lens_mean, 2),
                   "offset_width": w, "parallelism": "replicas" if world > 1 else "single",
                   "l2": f"inputs larger than L2 (arena {ab / 1e9:.2f} GB)"},
        "key_gbs": round(ss.text_bytes * args.steps * world / (ms / 1e3) / 1e9, 2),
        "roofline": roofline, "sort_roofline": sort_roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clocks.summary(), "tuning": tuning,
        "params": params,
        "stats": {k: v for k, v in st.as_dict().items()}, "kernels": per_kernel,
    }
    return out


# ---- text inputs: string starts found on the GPU, then the sort --------------------
TEXT_WORKLOADS = ("text_urls_50m", "suffixes_160m")


def text_workload(name, scale):
    """(text followed by 16 zero bytes, text length, mode of the device-resident
    steps, mode of the host-buffer steps, a function giving the text with the
    host mode's delimiters, number of strings, a function giving the uint64
    starts of the first m strings) for a text workload."""
    if name == "text_urls_50m":
        ss = pyssort.gen_urls(int(50_000_000 * scale), 4096, 1.1, 2)
        tlen = ss.text_bytes

        def lines():
            t = ss.arena[:tlen].copy()
            t[t == 0] = ord("\n")
            return t
        return (ss.arena, tlen, pyssort.TEXT_RAW, pyssort.TEXT_LINES, lines, ss.n,
                lambda m: ss.offs[:m])
    tlen = int(160_000_000 * scale)
    text = pyssort.gen_repeat_text(tlen, n_repeats=max(1, int(2000 * scale)), seed=8)
    return (text, tlen, pyssort.TEXT_SUFFIXES, pyssort.TEXT_SUFFIXES, lambda: text[:tlen], tlen,
            lambda m: np.arange(m, dtype=np.uint64))


def run_text(args, rank, world, local_rank, dist):
    """Whole-text sorts: a step finds the string starts of a resident text
    (ssort_text_offsets_device) and sorts them (ssort_sort_device); e2e is
    ssort_sort_text_host on the text in pinned host memory (copy in, find,
    sort, sorted starts out)."""
    import torch
    torch.cuda.set_device(local_rank)
    dev = f"cuda:{local_rank}"
    text, tlen, mode, host_mode, host_text, n, starts_of = text_workload(args.workload, args.scale)
    w = 4  # both texts are shorter than 2^32 bytes
    d_text = torch.from_numpy(text).to(dev)
    d_offs = torch.empty(n, dtype=torch.int32, device=dev)
    d_perm = torch.empty(n, dtype=torch.int32, device=dev)
    d_lcp = torch.empty(n, dtype=torch.int32, device=dev)
    sorter = pyssort.Sorter(local_rank)
    apply_params(sorter, args)
    stream = torch.cuda.Stream(device=local_rank)

    def step():
        m = sorter.text_offsets_device(d_text, tlen, mode, d_offs, w, n,
                                       stream=stream.cuda_stream)
        sorter.sort_device(d_text, tlen + 16, d_offs, w, m, d_perm, d_lcp,
                           stream=stream.cuda_stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    clocks = Clocks(local_rank)
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    time.sleep(0.3)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        dist.barrier()
    sorter.set_profiling(True)
    for _ in range(args.steps):
        step()
    torch.cuda.synchronize()
    ktimes = sorter.kernel_times()
    sorter.set_profiling(False)
    st = sorter.stats()
    ms = max_over_ranks(dist, ms, dev)

    e2e = None
    if not args.no_e2e:
        h_text = torch.empty(tlen, dtype=torch.uint8, pin_memory=True)
        h_text.numpy()[:] = host_text()
        h_out = torch.empty(n, dtype=torch.int64, pin_memory=True)
        ht, ho = h_text.numpy(), h_out.numpy().view(np.uint64)
        sorter.sort_text(ht, host_mode, with_lcp=False, out=ho)  # warm the staging buffers
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            sorter.sort_text(ht, host_mode, with_lcp=False, out=ho)
        e2e_s = max_over_ranks(dist, time.perf_counter() - t0, dev)
        e2e = {"value": job_rate(n, args.steps, world, e2e_s), "unit": UNIT,
               "h2d_bytes_per_step": int(tlen), "d2h_bytes_per_step": int(n * 8),
               "ms_per_step": 1000 * e2e_s / args.steps,
               "api": "ssort_sort_text_host (pinned host text), sorted string starts read back"}
    clocks.stop()
    if rank != 0:
        return None

    peak, peak_kind = peaks()
    kb = kernel_bytes(st, w)
    # text scan: count reads the text; starts reads it again and writes the
    # offsets; suffix mode writes the offsets only
    kb.update({"text_count": tlen, "text_starts": tlen + n * w, "iota_offs": n * w})
    per_kernel = {}
    for name, (kms, launches) in ktimes.items():
        entry = {"ms_total": round(kms, 4), "launches": int(launches),
                 "ms_per_step": round(kms / args.steps, 4)}
        if name in kb and kms > 0:
            entry["algorithmic_bytes_per_step"] = int(kb[name])
            entry["gbs"] = round(kb[name] * args.steps / (kms / 1e3) / 1e9, 1)
        per_kernel[name] = entry
    timed = {k: v for k, v in per_kernel.items() if "gbs" in v}
    dom = max(timed, key=lambda k: timed[k]["ms_total"]) if timed else None
    roofline = None
    if dom:
        d = per_kernel[dom]
        per_launch_bytes = kb[dom] * args.steps / d["launches"]
        per_launch_s = d["ms_total"] / 1e3 / d["launches"]
        ach = per_launch_bytes / per_launch_s / 1e9
        roofline = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                    "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 4),
                    "traffic": None, "algorithmic_bytes_per_launch": int(per_launch_bytes),
                    "launch_ms": round(per_launch_s * 1e3, 4)}
    lcp = d_lcp.cpu().numpy().view(np.uint32)
    live8 = intrinsic_live(lcp, n)
    sort_bytes = sort_algorithmic_bytes(live8, n, w)
    sort_s = ms / 1e3 / args.steps
    sort_roof = {"bound": "hbm", "algorithmic_bytes_per_sort": int(sort_bytes),
                 "achieved": round(sort_bytes / sort_s / 1e9, 1), "peak": peak,
                 "frac": round(sort_bytes / sort_s / 1e9 / peak, 4),
                 "live_per_8byte_round_first16": live8[:16], "rounds_8byte": len(live8),
                 "formula": "sum_r m_r*(4+W+8+24) + n*8, m_r from the LCP array"}
    launches = sum(v["launches"] * (3 if k == "scan" else 1) for k, v in per_kernel.items())
    cpu = None
    if not args.no_cpu and world == 1:
        cpu = cpu_baseline(args.workload, TextSample(text, starts_of, n))
    return {
        "metric": METRIC, "value": job_rate(n, args.steps, world, ms / 1e3), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": args.workload, "description": DESCRIPTIONS[args.workload],
                   "n_strings": n, "text_bytes": tlen, "offset_width": w,
                   "max_lcp": int(lcp.max()) if n else 0,
                   "mean_lcp": round(float(lcp.mean()), 2) if n else 0,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": f"inputs larger than L2 (text {tlen / 1e9:.2f} GB, offsets "
                         f"{n * w / 1e9:.2f} GB)"},
        "key_gbs": round(tlen * args.steps * world / (ms / 1e3) / 1e9, 2),
        "roofline": roofline, "sort_roofline": sort_roof, "cpu_baseline": cpu, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clocks.summary(),
        "stats": {k: v for k, v in st.as_dict().items()}, "kernels": per_kernel,
    }


class TextSample:
    """The first strings of a text workload in the form the CPU timers read:
    the padded text as the arena and the strings' starts as uint64 offsets."""

    def __init__(self, text, starts_of, n):
        self.arena = text
        self.n = n
        self._starts_of = starts_of
        self.offs = None

    def first(self, m):
        self.offs = np.ascontiguousarray(self._starts_of(m), dtype=np.uint64)
        return self


BATCH_WAVE_STRINGS = 200_000_000  # strings per wave of the full batched list


def check_instance(arena, offs, perm, lcp):
    """Problems with one sorted instance (empty string when it is right):
    perm must be a permutation, the strings in byte order with equal strings
    in index order (the stable order), and lcp[k] the common prefix length
    of neighbours k-1 and k (lcp[0] = 0)."""
    n = len(offs)
    if len(perm) != n or not np.array_equal(np.sort(perm), np.arange(n, dtype=np.uint32)):
        return "not a permutation"
    buf = arena.tobytes() if not isinstance(arena, bytes) else arena

    def s(i):
        o = int(offs[i])
        return buf[o:buf.index(b"\0", o)]
    prev = None
    for k in range(n):
        cur = s(int(perm[k]))
        if k == 0:
            if lcp[0] != 0:
                return "lcp[0] != 0"
        else:
            if prev > cur or (prev == cur and perm[k - 1] > perm[k]):
                return f"order broken at {k}"
            m = 0
            while m < len(prev) and m < len(cur) and prev[m] == cur[m]:
                m += 1
            if lcp[k] != m:
                return f"lcp wrong at {k}"
        prev = cur
    return ""


def run_batch_full(args):
    """The whole batched instance list, not the 1.5e9-byte subset: 20,000
    instances (about 4.0e9 strings, 1.2e11 key bytes; far more than one
    sort's 32-bit positions and the device memory), streamed through one GPU
    in waves of consecutive instances of up to BATCH_WAVE_STRINGS strings.
    Each wave is one batched call; a host thread generates the next wave
    while the GPU sorts the current one.  `value` counts device time (CUDA
    events around each batched call); wall time (generation, copies,
    checks) is reported beside it.  Two instances of every wave are checked
    for order, stability and every LCP entry (check_instance)."""
    import queue
    import threading as th

    import torch
    torch.cuda.set_device(0)
    params = pyssort.batch_instance_params(20000, 5)
    if args.scale < 1.0:
        params = params[:max(1, int(len(params) * args.scale))]
    waves, cur, m = [], [], 0
    for p in params:
        if cur and m + p[0] > BATCH_WAVE_STRINGS:
            waves.append(cur)
            cur, m = [], 0
        cur.append(p)
        m += p[0]
    if cur:
        waves.append(cur)
    q = queue.Queue(maxsize=1)

    def producer():
        for k, wp in enumerate(waves):
            q.put((k, wp, pyssort.gen_instances(wp, seed=1000 + k)))
        q.put(None)

    prod = th.Thread(target=producer, daemon=True)
    sorter = pyssort.Sorter(0)
    apply_params(sorter, args)
    stream = torch.cuda.Stream()
    rng = np.random.default_rng(9)
    clocks = Clocks(0)
    clocks.start()
    t0 = time.perf_counter()
    prod.start()
    dev_ms = 0.0
    tot_n = tot_bytes = tot_inst = checked = 0
    launches = []
    while True:
        item = q.get()
        if item is None:
            break
        k, wp, ss = item
        n, ninst = ss.n, len(wp)
        d_arena = torch.from_numpy(ss.arena).cuda()
        d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
        d_inst = torch.from_numpy(ss.inst_start.view(np.int32)).cuda()
        d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
        d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sorter.sort_batch_device(d_arena, ss.arena.nbytes, d_offs, 8, n, d_inst, ninst, d_perm,
                                 d_lcp, stream=stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        dev_ms += e0.elapsed_time(e1)
        # two instances of the wave (of at most 50,000 strings) checked
        st = ss.inst_start
        small = [i for i in range(ninst) if 2 <= int(st[i + 1]) - int(st[i]) <= 50_000]
        for i in rng.choice(small, size=min(2, len(small)), replace=False) if small else []:
            lo, hi = int(st[i]), int(st[i + 1])
            gp = d_perm[lo:hi].cpu().numpy().view(np.uint32)
            gl = d_lcp[lo:hi].cpu().numpy().view(np.uint32)
            bad = check_instance(ss.arena, ss.offs[lo:hi], gp, gl)
            if bad:
                raise RuntimeError(f"wave {k} instance {i}: {bad}")
            checked += 1
        tot_n += n
        tot_bytes += ss.text_bytes
        tot_inst += ninst
        launches.append(n)
        del d_arena, d_offs, d_inst, d_perm, d_lcp, ss
    wall = time.perf_counter() - t0
    prod.join()
    clocks.stop()
    sorter.close()
    return {
        "metric": METRIC, "value": tot_n / (dev_ms / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": len(waves), "warmup": 0, "ms_per_step": dev_ms / len(waves),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": "batch_c4_full",
                   "description": "the full list: " + DESCRIPTIONS["batch_c4"].split(";")[0] +
                                  f"; {len(params)} instances in {len(waves)} waves of at most "
                                  f"{BATCH_WAVE_STRINGS:,} strings, one batched call per wave; "
                                  "seeds 5 (list), 1000 + wave (strings)",
                   "n_instances": tot_inst, "n_strings": tot_n, "key_bytes": tot_bytes,
                   "parallelism": "single", "l2": "inputs larger than L2 (GBs per wave)"},
        "key_gbs": round(tot_bytes / (dev_ms / 1e3) / 1e9, 2),
        "device_s": round(dev_ms / 1e3, 3), "wall_s": round(wall, 2),
        "wall_strings_per_s": tot_n / wall,
        "wall_note": "wall time includes host generation of every wave (overlapped with the "
                     "sorts), the pageable host-to-device copies and the oracle checks",
        "instances_checked_against_oracle": checked, "clocks": clocks.summary(),
    }


def run_batch(args):
    """Batched form vs plain form on the same GPU: one ssort_sort_batch_device
    call over all instances vs one ssort_sort_device call per instance."""
    import torch
    torch.cuda.set_device(0)
    params = pyssort.batch_instance_params(20000, 5, key_byte_limit=1.5e9 * args.scale)
    ss = pyssort.gen_instances(params, seed=4)
    n, k = ss.n, len(params)
    d_arena = torch.from_numpy(ss.arena).cuda()
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
    d_inst = torch.from_numpy(ss.inst_start.view(np.int32)).cuda()
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    sorter = pyssort.Sorter(0)
    apply_params(sorter, args)
    stream = torch.cuda.Stream()
    ab = ss.arena.nbytes

    def batched():
        sorter.sort_batch_device(d_arena, ab, d_offs, 8, n, d_inst, k, d_perm, d_lcp,
                                 stream=stream.cuda_stream)

    starts = [int(x) for x in ss.inst_start]

    def plain():
        for i in range(k):
            lo, hi = starts[i], starts[i + 1]
            if hi > lo:
                sorter.sort_device(d_arena, ab, d_offs.data_ptr() + 8 * lo, 8, hi - lo,
                                   d_perm.data_ptr() + 4 * lo, d_lcp.data_ptr() + 4 * lo,
                                   stream=stream.cuda_stream)

    def timed(fn, steps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(steps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / steps

    for _ in range(args.warmup):
        batched()
    clocks = Clocks(0)
    clocks.start()
    time.sleep(0.3)
    ms_b = timed(batched, args.steps)
    st = sorter.stats()
    # launches of one batched call (the scan is three kernels per launch)
    sorter.set_profiling(True)
    batched()
    torch.cuda.synchronize()
    kt = sorter.kernel_times()
    sorter.set_profiling(False)
    launches_per_call = int(sum(v[1] * (3 if k == "scan" else 1) for k, v in kt.items()))
    plain()
    ms_p = timed(plain, max(1, min(args.steps, 3)))
    clocks.stop()
    return {
        "metric": METRIC, "value": n / (ms_b / 1e3), "unit": UNIT, "n_gpus": 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_b,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": "batch_c4", "description": DESCRIPTIONS["batch_c4"],
                   "n_instances": k, "n_strings": n, "key_bytes": int(ss.text_bytes),
                   "parallelism": "single", "l2": f"inputs larger than L2 (arena {ab / 1e9:.2f} GB)"},
        "key_gbs": round(ss.text_bytes / (ms_b / 1e3) / 1e9, 2),
        "plain": {"value": n / (ms_p / 1e3), "unit": UNIT, "ms_per_step": ms_p,
                  "calls_per_step": k},
        "batched_vs_plain": round(ms_p / ms_b, 2), "launches_per_call": launches_per_call,
        "clocks": clocks.summary(), "stats": st.as_dict(),
    }


# ---- serving: Poisson request stream ------------------------------------------------
class RequestPool:
    """Distinct sort requests in pinned host memory: string counts log-uniform
    in [1,000, 5,000,000], strings as in the batched workload.  Each request's
    bytes start 16-byte aligned in one arena; its uint32 offsets are relative
    to that start; perm/lcp output buffers per request."""

    def __init__(self, npool, seed=6):
        import torch
        params = pyssort.batch_instance_params(npool, seed, lo=1000, hi=5_000_000)
        ss = pyssort.gen_instances(params, seed=seed + 1)
        spans = []
        for i in range(len(params)):
            lo, hi = int(ss.inst_start[i]), int(ss.inst_start[i + 1])
            a0 = int(ss.offs[lo])
            a1 = int(ss.offs[hi]) if hi < ss.n else ss.text_bytes
            spans.append((lo, hi, a0, a1))
        total = sum((a1 - a0 + 15) // 16 * 16 for _, _, a0, a1 in spans) + 16
        self.arena = torch.zeros(total, dtype=torch.uint8, pin_memory=True).numpy()
        u32 = lambda m: torch.empty(max(m, 1), dtype=torch.int32,  # noqa: E731
                                    pin_memory=True).numpy().view(np.uint32)
        self.offs, self.perm, self.lcp = u32(ss.n), u32(ss.n), u32(ss.n)
        self.reqs = []
        at = 0
        for lo, hi, a0, a1 in spans:
            nb = a1 - a0
            self.arena[at:at + nb] = ss.arena[a0:a1]
            self.offs[lo:hi] = ss.offs[lo:hi] - np.uint64(a0)
            self.reqs.append({"at": at, "nb": nb, "lo": lo, "m": hi - lo})
            at += (nb + 15) // 16 * 16
        self.n = ss.n
        self.key_bytes = ss.text_bytes
        self.dev = None

    def host(self, k):
        r = self.reqs[k]
        lo, m = r["lo"], r["m"]
        return (self.arena[r["at"]:r["at"] + r["nb"]], self.offs[lo:lo + m],
                self.perm[lo:lo + m], self.lcp[lo:lo + m])

    def to_device(self):
        """Device copies of the pool (inputs resident in HBM) plus device
        output buffers; returns base addresses."""
        import torch
        d_arena = torch.from_numpy(self.arena).cuda()
        d_offs = torch.from_numpy(self.offs.view(np.int32)).cuda()
        d_perm = torch.empty_like(d_offs)
        d_lcp = torch.empty_like(d_offs)
        self.dev = (d_arena, d_offs, d_perm, d_lcp)
        return [t.data_ptr() for t in self.dev]

    def device(self, k):
        a, o, p, c = [t.data_ptr() for t in self.dev]
        r = self.reqs[k]
        lo = r["lo"]
        return a + r["at"], r["nb"], o + 4 * lo, r["m"], p + 4 * lo, c + 4 * lo


def _arrivals(nreq, rate, npool, seed):
    u = pyssort.uniform_doubles(2 * nreq, seed)
    gaps = -np.log1p(-u[:nreq]) / rate
    t = np.cumsum(gaps)
    t -= t[0]
    picks = np.minimum((u[nreq:] * npool).astype(np.int64), npool - 1)
    return t, picks


def _wait_until(t0, t):
    while True:
        d = t - (time.perf_counter() - t0)
        if d <= 0:
            return
        time.sleep(d if d > 2e-3 else 0)


def _lat_summary(lat_s, strings, span_s, key_bytes):
    a = np.asarray(lat_s) * 1e3
    return {"p50_ms": round(float(np.percentile(a, 50)), 3),
            "p99_ms": round(float(np.percentile(a, 99)), 3),
            "p999_ms": round(float(np.percentile(a, 99.9)), 3),
            "max_ms": round(float(a.max()), 3),
            "strings_per_s": strings / span_s, "key_gbs": round(key_bytes / span_s / 1e9, 2),
            "req_per_s": round(len(a) / span_s, 1), "span_s": round(span_s, 3)}


def serve_stream(srv, pool, arrivals, picks, resident=False):
    """Open-loop stream through the request server: each request is submitted
    at its arrival time; latency runs from arrival to the step that reports
    it done (results in host memory, or in device memory when resident)."""
    n = len(arrivals)
    lat = np.zeros(n)
    owner = {}
    nxt = done = strings = kb = 0
    t0 = time.perf_counter()
    while done < n:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now:
            k = picks[nxt]
            if resident:
                a, nb, o, m, p, c = pool.device(k)
                rid = srv.submit_ptr(a, nb, o, 4, m, p, c)
            else:
                a, o, p, c = pool.host(k)
                rid, _, _ = srv.submit(a, o, perm=p, lcp=c)
            owner[rid] = nxt
            nxt += 1
        ids = srv.step()
        t = time.perf_counter() - t0
        for rid in ids:
            k = owner.pop(rid)
            lat[k] = t - arrivals[k]
            r = pool.reqs[picks[k]]
            strings += r["m"]
            kb += r["nb"]
            done += 1
        if not ids and nxt < n and not owner:
            _wait_until(t0, arrivals[nxt])
    span = time.perf_counter() - t0
    return _lat_summary(lat, strings, span, kb)


def plain_stream(sorter, pool, arrivals, picks, resident=False):
    """The same stream through the plain entry points, one request at a time
    in arrival order: ssort_sort_host (copy in, sort, copy out), or
    ssort_sort_device on the resident copy."""
    n = len(arrivals)
    lat = np.zeros(n)
    strings = kb = 0
    t0 = time.perf_counter()
    for j in range(n):
        _wait_until(t0, arrivals[j])
        k = picks[j]
        if resident:
            a, nb, o, m, p, c = pool.device(k)
            sorter.sort_device(a, nb, o, 4, m, p, c)
        else:
            a, o, p, c = pool.host(k)
            sorter.sort_host(a, o, perm=p, lcp=c)
        lat[j] = time.perf_counter() - t0 - arrivals[j]
        r = pool.reqs[k]
        strings += r["m"]
        kb += r["nb"]
    span = time.perf_counter() - t0
    return _lat_summary(lat, strings, span, kb)


def run_serve(args):
    import torch
    torch.cuda.set_device(0)
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    # Fresh requests: every request of every rate's stream is a distinct,
    # newly generated one (up to SERVE_FRESH_CAP in all, a host- and
    # device-memory bound); otherwise the streams draw from a pool.
    fresh = getattr(args, "serve_fresh", False)
    need = args.serve_requests * len(rates)
    pool = RequestPool(min(need, SERVE_FRESH_CAP) if fresh else args.serve_pool)
    fresh = fresh and len(pool.reqs) >= need
    pool.to_device()
    budget = int(args.serve_budget_gb * 1e9)
    srv = pyssort.Server(budget, args.serve_max_strings)
    sorter = pyssort.Sorter(0)
    # warm-up: the largest pool requests once through each path, largest
    # first so that the plain context's buffers reach their final size
    order = np.array(sorted(range(len(pool.reqs)), key=lambda k: -pool.reqs[k]["m"])[:64])
    w_arr = np.zeros(len(order))
    for _ in range(max(1, args.warmup)):
        for resident in (False, True):
            serve_stream(srv, pool, w_arr, order, resident)
    for resident in (False, True):
        plain_stream(sorter, pool, w_arr, order, resident)
    clocks = Clocks(0)
    clocks.start()
    sweeps = {}
    for resident in (False, True):
        rows = []
        for i, rate in enumerate(rates):
            arr, picks = _arrivals(args.serve_requests, rate, len(pool.reqs), 100 + i)
            if fresh:  # distinct requests, none replayed
                picks = np.arange(i * args.serve_requests, (i + 1) * args.serve_requests)
            served = serve_stream(srv, pool, arr, picks, resident)
            plain = plain_stream(sorter, pool, arr, picks, resident)
            rows.append({"rate_req_s": rate, "served": served, "plain": plain,
                         "served_vs_plain": round(served["strings_per_s"] /
                                                  plain["strings_per_s"], 2)})
        sweeps["resident" if resident else "host"] = rows
    clocks.stop()
    info = srv.info()
    srv.close()
    best_h = max(sweeps["host"], key=lambda r: r["served"]["strings_per_s"])
    best_d = max(sweeps["resident"], key=lambda r: r["served"]["strings_per_s"])
    return {
        "metric": "served sort throughput (strings/s) with p50/p99/p99.9 latency",
        "value": best_d["served"]["strings_per_s"], "unit": UNIT, "n_gpus": 1,
        "steps": args.serve_requests, "warmup": args.warmup,
        "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": "serve_c5", "description": DESCRIPTIONS["serve_c5"],
                   "requests_per_rate": args.serve_requests, "pool_requests": len(pool.reqs),
                   "fresh_requests": bool(fresh),
                   "pool_strings": pool.n, "pool_key_bytes": pool.key_bytes,
                   "arena_budget_bytes": budget, "max_strings": args.serve_max_strings,
                   "parallelism": "single",
                   "l2": "inputs larger than L2 (pool of requests, GBs)"},
        "e2e": {"value": best_h["served"]["strings_per_s"], "unit": UNIT,
                "note": "requests from pinned host buffers; copies in and out inside each "
                        "request's latency"},
        "sweep_resident": sweeps["resident"], "sweep_host": sweeps["host"],
        "server": info, "clocks": clocks.summary(),
    }

def _ref_lib():
    p = os.path.join(ROOT, "oracle", "_ref", "libref.so")
    if not os.path.exists(p):
        return None
    L = ctypes.CDLL(p)
    L.ref_time_sort.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_size_t]
    L.ref_time_sort.restype = ctypes.c_double
    return L


def _port_lib():
    L = ctypes.CDLL(os.path.join(ROOT, "oracle", "liboracle.so"))
    L.oracle_sort_arena.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                    ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p]
    return L


def time_dropin(ss, n, steps):
    """The drop-in as the reference's own driver calls it: msd_gpu(strings, n)
    through r->f of the reference's routine registry (sortstring's run(),
    src/sortstring.c:424-451), on a pointer array into the workload's arena
    in ordinary (pageable) host memory.  The pointer array is built outside
    the timed call, as sortstring builds it while reading its input.  One
    untimed call first (the routine's context and staging buffers)."""
    p = os.path.join(ROOT, "oracle", "_ref", "libref_dropin.so")
    if not os.path.exists(p):
        return None
    L = ctypes.CDLL(p)
    L.ref_time_sort.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_size_t]
    L.ref_time_sort.restype = ctypes.c_double
    if L.ref_time_sort(b"msd_gpu", ss.arena.ctypes.data, ss.offs.ctypes.data, n) < 0:
        return None
    ts = [L.ref_time_sort(b"msd_gpu", ss.arena.ctypes.data, ss.offs.ctypes.data, n)
          for _ in range(steps)]
    t = statistics.median(ts)
    return {"value": n / t, "unit": UNIT, "ms_per_step": round(1000 * t, 3), "steps": steps,
            "api": "msd_gpu(unsigned char **, size_t) through the reference registry's r->f",
            "h2d_bytes_per_step": int(ss.text_bytes + n * (4 if ss.text_bytes < 2**32 else 8)),
            "d2h_bytes_per_step": int(n * 8)}  # sorted 8-byte offsets into the span


def time_cpu_sort(ss, m):
    """Seconds for one sort of the first m strings: the reference's msd_CE6
    timed around its routine call, or the oracle port when the reference
    library is absent.  Returns (seconds, kind)."""
    L = _ref_lib()
    if L is not None:
        s = L.ref_time_sort(b"msd_CE6", ss.arena.ctypes.data, ss.offs.ctypes.data, m)
        if s < 0:
            raise RuntimeError("reference sort failed")
        return s, "reference"
    P = _port_lib()
    perm = np.empty(m, dtype=np.uint32)
    t0 = time.perf_counter()
    P.oracle_sort_arena(ss.arena.ctypes.data, ss.offs.ctypes.data, 8, m, perm.ctypes.data, None)
    return time.perf_counter() - t0, "port"


def instance_params(workload, budget):
    """(params, seed) of the first instances of the batched or served
    workload's list, up to about `budget` strings (a bounded sample)."""
    if workload == "batch_c4":
        params = pyssort.batch_instance_params(20000, 5, key_byte_limit=1.5e9)
        seed = 4
    else:
        params = pyssort.batch_instance_params(64, 6, lo=1000, hi=5_000_000)
        seed = 7
    take, total = [], 0
    for p in params:
        if take and total + p[0] > budget:
            break
        take.append(p)
        total += p[0]
    return take, seed


def instance_sample(workload, budget):
    take, seed = instance_params(workload, budget)
    return pyssort.gen_instances(take, seed=seed)


def time_cpu_instances(ss):
    """Seconds for sorting every instance of ss one after another with the
    reference's msd_CE6 (or the oracle port).  Returns (seconds, kind)."""
    L = _ref_lib()
    total, kind = 0.0, "reference" if L is not None else "port"
    P = None if L is not None else _port_lib()
    for i in range(len(ss.inst_start) - 1):
        lo, hi = int(ss.inst_start[i]), int(ss.inst_start[i + 1])
        if hi - lo < 2:
            continue
        op = ss.offs.ctypes.data + 8 * lo
        if L is not None:
            t = L.ref_time_sort(b"msd_CE6", ss.arena.ctypes.data, op, hi - lo)
            if t < 0:
                raise RuntimeError("reference sort failed")
            total += t
        else:
            perm = np.empty(hi - lo, dtype=np.uint32)
            t0 = time.perf_counter()
            P.oracle_sort_arena(ss.arena.ctypes.data, op, 8, hi - lo, perm.ctypes.data, None)
            total += time.perf_counter() - t0
    return total, kind


# ---- all host cores on independent instances (separate processes) -----------------
_worker_ss = None


def _instances_worker_init(params, seed):
    """Each worker process generates the same instance list (seeded) once."""
    global _worker_ss
    sys.path.insert(0, os.path.join(ROOT, "string-sorting_b200"))
    import pyssort as _p
    _worker_ss = _p.gen_instances(params, seed=seed)


def _instances_worker_sort(ids):
    """Wall seconds for sorting instances `ids` of the worker's list with
    msd_CE6 one after another (the pointer arrays are built outside)."""
    L = _ref_lib()
    ss = _worker_ss
    total = 0.0
    for i in ids:
        lo, hi = int(ss.inst_start[i]), int(ss.inst_start[i + 1])
        if hi - lo >= 2:
            t = L.ref_time_sort(b"msd_CE6", ss.arena.ctypes.data, ss.offs.ctypes.data + 8 * lo,
                                hi - lo)
            if t < 0:
                raise RuntimeError("reference sort failed")
            total += t
    return total


class AllCoreInstances:
    """msd_CE6 on independent instances across every host core, one process
    per core (msd_CE3..CE8 keep function-static bucket arrays, so they are not
    reentrant and cannot share a process, src/msd_ce.cpp:392).  The instances
    are dealt to the workers largest first; a step's time is the slowest
    worker's.  Spawned processes: safe after the parent has used the GPU."""

    def __init__(self, params, seed, procs=None):
        import multiprocessing as mp
        self.procs = procs or os.cpu_count() or 1
        self.counts = [p[0] for p in params]
        order = sorted(range(len(params)), key=lambda i: -params[i][0])
        load = [0] * self.procs
        self.assign = [[] for _ in range(self.procs)]
        for i in order:
            k = min(range(self.procs), key=lambda j: load[j])
            self.assign[k].append(i)
            load[k] += params[i][0]
        self.pool = mp.get_context("spawn").Pool(self.procs, _instances_worker_init,
                                                 (params, seed))

    def step(self):
        return max(self.pool.map(_instances_worker_sort, self.assign, chunksize=1))

    def close(self):
        self.pool.close()
        self.pool.join()


# The reference's CPU routines timed beside the GPU sort (name, cores used,
# note).  msd_CE6 is the oracle; msd_CE7/CE8 share a sortedness shortcut that
# mis-sorts segments of >= 65,536 strings whose 2-byte keys are non-increasing
# but not all equal (src/msd_ce.cpp:452,529), so CE8 is timed but flagged.
CPU_ROUTINES = (
    ("msd_CE6", "stable MSD radix sort, 16-bit digits for >= 65,536 strings "
                "(src/msd_ce.cpp:367-419); the oracle"),
    ("msd_CE2", "stable MSD radix sort, 8-bit digits, reentrant (src/msd_ce.cpp:143-178)"),
    ("multikey_cache8", "multikey quicksort with an 8-byte cache (src/multikey_cache.cpp:231-238)"),
    ("multikey_cache4", "multikey quicksort with a 4-byte cache (src/multikey_cache.cpp:231-238)"),
    ("burstsort_vector", "burstsort with vector buckets (src/burstsort.cpp:290-299)"),
    ("msd_CE8", "FLAGGED: mis-sorts non-increasing 2-byte keys in segments >= 65,536 "
                "(src/msd_ce.cpp:529); timed only"),
    ("parallel_msd_radix_sort", "multicore MSD radix sort (external/"
                                "parallel_string_radix_sort.cpp), OpenMP over all host threads"),
)


def cpu_routines(ss, m, reps=5):
    """Every routine of CPU_ROUTINES on the first m strings of ss, median of
    `reps` runs each (fresh pointer array per run), through the reference's
    own routine registry.  None when the reference library is absent."""
    L = _ref_lib()
    if L is None:
        return None
    out = {}
    for name, note in CPU_ROUTINES:
        ts = []
        for _ in range(reps):
            t = L.ref_time_sort(name.encode(), ss.arena.ctypes.data, ss.offs.ctypes.data, m)
            if t < 0:
                ts = None
                break
            ts.append(t)
        if not ts:
            out[name] = {"unavailable": "not registered in the reference library"}
            continue
        t = statistics.median(ts)
        cores = os.cpu_count() if name == "parallel_msd_radix_sort" else 1
        out[name] = {"value": m / t, "unit": UNIT, "seconds_median": round(t, 4),
                     "runs": reps, "cores": cores, "note": note}
    return out


def cpu_baseline(workload, ss, reps=5):
    m = min(ss.n, CPU_SAMPLE.get(workload, 2_000_000))
    if isinstance(ss, TextSample):
        ss.first(m)
    ts = []
    kind = None
    for _ in range(reps):
        t, kind = time_cpu_sort(ss, m)
        ts.append(t)
    t = statistics.median(ts)
    out = {"value": m / t, "unit": UNIT, "cores": 1, "kind": kind,
           "routine": "msd_CE6" if kind == "reference" else "oracle port of msd_CE6",
           "sample": f"first {m:,} strings of {workload}, median of {reps} runs "
                     f"({t:.3f} s each), single thread",
           "host": {"cpu": cpu_model(), "nproc": os.cpu_count()}}
    if kind == "reference":
        out["routines"] = cpu_routines(ss, m, reps)
    return out



# ---- the other configurations, measured in the same run ---------------------------
def plain_config_summary(workload, steps, warmup, no_cpu):
    """One more plain configuration measured beside the headline: strings/s
    from device-resident inputs (CUDA events on the sort's stream), the
    whole-sort roofline, the dominant kernel's roofline from a profiled pass,
    and msd_CE6 on a bounded sample of the same strings."""
    import torch
    ss = pyssort.WORKLOADS[workload]()
    n, w, ab = ss.n, ss.offs.dtype.itemsize, ss.arena.nbytes
    d_arena = torch.from_numpy(ss.arena).cuda()
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.Stream()
    with pyssort.Sorter(0) as sorter:
        def step():
            sorter.sort_device(d_arena, ab, d_offs, w, n, d_perm, d_lcp,
                               stream=stream.cuda_stream)
        for _ in range(warmup):
            step()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        sorter.set_profiling(True)
        for _ in range(steps):
            step()
        torch.cuda.synchronize()
        ktimes = sorter.kernel_times()
        sorter.set_profiling(False)
        st = sorter.stats()
    peak, peak_kind = peaks()
    kb = kernel_bytes(st, w)
    dom = max((k for k in ktimes if k in kb), key=lambda k: ktimes[k][0], default=None)
    roof = None
    if dom:
        kms, launches = ktimes[dom]
        ach = kb[dom] * steps / (kms / 1e3) / 1e9
        roof = {"kernel": dom, "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                "peak_kind": peak_kind, "unit": "GB/s", "frac": round(ach / peak, 4),
                "launch_ms": round(kms / launches, 4)}
    live8 = intrinsic_live(d_lcp.cpu().numpy().view(np.uint32), n)
    sb = sort_algorithmic_bytes(live8, n, w)
    out = {"workload": workload, "description": DESCRIPTIONS[workload], "n_strings": n,
           "value": n / (ms / 1e3), "unit": UNIT, "ms_per_step": round(ms, 4), "steps": steps,
           "warmup": warmup, "key_gbs": round(ss.text_bytes / (ms / 1e3) / 1e9, 2),
           "sort_roofline": {"algorithmic_bytes_per_sort": int(sb),
                             "achieved": round(sb / (ms / 1e3) / 1e9, 1), "peak": peak,
                             "frac": round(sb / (ms / 1e3) / 1e9 / peak, 4),
                             "frac_of_8tbs": round(sb / (ms / 1e3) / 1e9 / 8000, 4),
                             "live_per_8byte_round": live8[:8]},
           "roofline": roof,
           "kernels_ms_per_step": {k: round(v[0] / steps, 4) for k, v in sorted(
               ktimes.items(), key=lambda kv: -kv[1][0])[:8]},
           "stats": {k: st.as_dict()[k] for k in ("rounds", "partition_levels", "partitioned")}}
    if not no_cpu:
        out["cpu_baseline"] = cpu_baseline(workload, ss, reps=3)
    del d_arena, d_offs, d_perm, d_lcp
    torch.cuda.empty_cache()
    return out


def extra_configs(args):
    """The other configurations of the benchmark, each measured briefly in the
    default run so that one invocation reports all of them: the uniform 1 M
    and Zipf-words 100 M plain sorts, the batched-vs-plain ratio on the
    batched workload, and a two-rate serving sweep with latency percentiles."""
    import argparse as _ap
    import torch
    out = {}
    for wl in ("zipf_words_100m", "uniform_1m"):
        out[wl] = plain_config_summary(wl, 5, 3, args.no_cpu)
    b = run_batch(_ap.Namespace(scale=1.0, warmup=2, steps=3))
    out["batch_c4"] = {k: b[k] for k in ("value", "unit", "ms_per_step", "plain",
                                         "batched_vs_plain", "config", "launches_per_call")
                       if k in b}
    torch.cuda.empty_cache()
    sv = run_serve(_ap.Namespace(serve_rates="1000,20000", serve_pool=args.serve_pool,
                                 serve_requests=300, serve_budget_gb=args.serve_budget_gb,
                                 serve_max_strings=args.serve_max_strings, warmup=1,
                                 serve_fresh=True))
    out["serve_c5"] = {k: sv[k] for k in ("value", "unit", "config", "sweep_resident",
                                          "sweep_host") if k in sv}
    torch.cuda.empty_cache()
    return out


def run_reference(args, rank):
    if rank != 0:
        return None
    warm = None
    cores = 1
    pool = None
    same = False
    if args.workload in ("batch_c4", "batch_c4_full", "serve_c5"):
        # independent instances, each sorted alone by msd_CE6, spread over
        # every host core (one process per core)
        params, seed = instance_params("serve_c5" if args.workload == "serve_c5" else "batch_c4",
                                       16_000_000)
        ss = pyssort.gen_instances(params, seed=seed)
        m = ss.n
        kind0 = "reference" if _ref_lib() is not None else "port"
        if kind0 == "reference":
            pool = AllCoreInstances(params, seed)
            cores = pool.procs
            timer = lambda: (pool.step(), "reference")  # noqa: E731
        else:
            timer = lambda: time_cpu_instances(ss)  # noqa: E731
        sample = (f"the first {len(params)} instances ({m:,} strings) of the {args.workload} "
                  f"list per step, each sorted alone, on {cores} host cores (one process each)")
    elif args.workload in TEXT_WORKLOADS:
        text, _, _, _, _, n, starts_of = text_workload(args.workload, args.scale)
        m = min(n, CPU_SAMPLE[args.workload])
        ss = TextSample(text, starts_of, n).first(m)
        sample = f"first {m:,} strings of {args.workload} per step (pointers into the whole text)"
        timer = lambda: time_cpu_sort(ss, m)  # noqa: E731
    else:
        # The plain workloads: every timed step sorts the whole configuration
        # (the same strings the GPU arm sorts); warm-up steps sort the bounded
        # sample, which touches the same code and pages.
        ss = pyssort.WORKLOADS[args.workload](args.scale)
        m = ss.n
        ms_ = min(ss.n, CPU_SAMPLE.get(args.workload, 2_000_000))
        sample = (f"all {m:,} strings of {args.workload} per timed step (the full "
                  f"configuration); warm-up steps sort the first {ms_:,}")
        timer = lambda: time_cpu_sort(ss, m)  # noqa: E731
        warm = lambda: time_cpu_sort(ss, ms_)  # noqa: E731
        same = True
    if warm is None:
        warm = timer
    for _ in range(args.warmup):
        warm()
    total = 0.0
    kind = None
    timed = 0
    t_start = time.perf_counter()
    for _ in range(args.steps):
        t, kind = timer()
        total += t
        timed += 1
        # Bounded run: once the timed steps have taken REF_BUDGET_S, the
        # remaining steps are skipped (reported in steps_timed).
        if time.perf_counter() - t_start > REF_BUDGET_S:
            break
    if pool is not None:
        pool.close()
    v = m * timed / total
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "steps_timed": timed, "warmup": args.warmup,
        "ms_per_step": 1000 * total / timed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded generator, stand-in for the reference's text corpora)",
        "config": {"workload": args.workload, "description": DESCRIPTIONS.get(args.workload),
                   "n_strings": ss.n, "sample_strings": m, "same_config": same},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind,
                         "routine": "msd_CE6 (single-threaded by design: function-static "
                                    "bucket arrays, src/msd_ce.cpp:392)",
                         "sample": sample,
                         "host": {"cpu": cpu_model(), "nproc": os.cpu_count()}},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    if args.workload in ("batch_c4", "batch_c4_full", "serve_c5"):
        if rank == 0:
            fn = {"batch_c4": run_batch, "batch_c4_full": run_batch_full,
                  "serve_c5": run_serve}[args.workload]
            print(json.dumps(fn(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(local_rank)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                 device_id=torch.device(f"cuda:{local_rank}"))
        dist = tdist
    try:
        fn = run_text if args.workload in TEXT_WORKLOADS else run_ours
        out = fn(args, rank, world, local_rank, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()
    if (out is not None and world == 1 and args.workload == DEFAULT_WORKLOAD and
            args.scale == 1.0 and not args.no_extras):
        import gc
        gc.collect()
        out["configs"] = extra_configs(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
