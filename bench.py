#!/usr/bin/env python
"""Distance-index build benchmark (one JSON line on rank 0).

Workload: the plain index build at chromosome scale -- a synthetic sequence
graph of 5e7 backbone bases (SNP 1/1000, indel 1/5000 with geometric length
mean 4 capped at 50, 0.1 % of bubbles structural with length 100..2000, seed
42), adjacency in range CRS with uint32 columns, index = A^400 * (A+I)^200
(distance window [400, 600]).  A step is one complete index build.

  value    seconds per build with A already resident in HBM (device time over
           the timed steps, CUDA events on the library's stream, max over ranks)
  e2e      the same through the C ABI with host buffers: every step copies A
           from pinned host memory, builds, and copies the index back
  roofline the range-SpGEMM kernel (k_spgemm_rowmode, one pass per product):
           algorithmic bytes per product (read A and B once, write C once) / its
           mean duration, from CUDA-event spans around every launch in a second,
           instrumented repetition of the timed builds
  cpu_baseline the CPU restatement of the reference's bitvector SpGEMM path and
           index schedule (OpenMP, all host threads), one build of the whole
           graph; its index is also the oracle the GPU index is compared with
           ("parity": every rowmap word, entry and the nnz equal)
  secondary (N = 1) the other workloads, each with its own clock samples:
           membership queries against the resident index, the range-SpGEMM /
           SpAdd kernel microbenchmark, batched builds of 2,000 graphs, and the
           serving loop under Poisson arrivals

--impl reference times that CPU restatement alone (the reference's own
Kokkos/OpenMP build cannot be compiled: its submodules are absent), one build
of the whole graph per timed step.
With N GPUs each rank builds its own graph (seed 42 + rank): the index is
block-diagonal over independent components, so ranks share no data.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0
L2_BYTES = 126 * 2**20
# DRAM bytes (read + write) per C row of the row kernel, mean of the three
# launches of the row kernel's ncu capture under profiles/ (10,019,292-row
# graph): traffic scales with the rows of the product
ROWMODE_TRAFFIC_BYTES_PER_ROW = (487831040 + 323487744 + 326833408 +
                                 154045184 + 137517312 + 142550272) / 3 / 10019292
QUERY_ALG_BYTES = 33  # pair 8 B, two rowmap words 16 B, one range 8 B, answer 1 B
QUERY_SECTOR_BYTES = 73  # two 32-byte sectors (row pointers, range), the pair, the answer


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n-backbone", type=int, default=50_000_000)
    p.add_argument("--dmin", type=int, default=400)
    p.add_argument("--dmax", type=int, default=600)
    p.add_argument("--seed", type=int, default=42)
    p.add_argument("--no-cpu-baseline", action="store_true",
                   help="skip the CPU build of the whole graph (and with it the parity check)")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-secondary", action="store_true", help="headline build only")
    p.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                   help="a context option (dvg_set_option) for the run; repeatable")
    p.add_argument("--workload", choices=["build", "batch", "spgemm", "serve", "adjacency", "query"],
                   default="build",
                   help="build: the plain chromosome-scale index build (the headline) followed by the "
                        "secondary workloads; batch: 2,000 mixed-size graphs in one batched build vs "
                        "back-to-back single builds; spgemm: range_spgemm / range_spadd alone on banded "
                        "2^24-row matrices; serve: the request loop under Poisson arrivals; query: membership "
                        "queries against the resident chromosome-scale index")
    p.add_argument("--graphs", type=int, default=2000, help="batch: number of graphs")
    p.add_argument("--kernels", default="automatic,tile-staged,row+levels,spadd",
                   help="spgemm: the kernels to time, a comma list of automatic, tile-staged, row+levels, spadd")
    p.add_argument("--log2-rows", type=int, default=24, help="spgemm: rows of the banded operands, as a power of two")
    p.add_argument("--rate", type=float, default=0.0, help="serve: arrivals per second (0: sweep)")
    p.add_argument("--requests", type=int, default=1000, help="serve: requests per rate")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, devices):
        self.devices = devices
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", ",".join(map(str, self.devices)), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.tmp, stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.tmp is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.tmp.flush()
        rows = []
        with open(self.tmp.name) as f:
            for ln in f:
                parts = [x.strip() for x in ln.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock samples"]}
        sm = [float(r[1]) for r in rows]
        mx = max(float(r[2]) for r in rows)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": reasons, "samples": len(rows),
                "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())
                if any(r[3].replace(".", "").isdigit() for r in rows) else None}


def graph(n_backbone, seed):
    from diverg_b200 import gen
    spec = gen.chromosome_graph_spec(n_backbone, seed=seed)
    return gen.graph_adjacency(spec)


def omat(m):
    from oracle import pyoracle as orc
    import numpy as np
    return orc.OMat(m.numRows(), m.numCols(), np.asarray(m.rowmap, dtype=np.uint64), m.entries, m.nnz())


def cpu_build(a, dmin, dmax):
    """One index build of `a` by the CPU restatement of the reference's path
    (bitvector SpGEMM, the reference's squaring schedule, OpenMP on every host
    thread): (seconds, the index)."""
    from oracle import pyoracle as orc
    oa = omat(a)
    t = time.perf_counter()
    idx = orc.dindex(oa, dmin, dmax, algo="hbv")
    return time.perf_counter() - t, idx


def cpu_kind_note():
    return ("CPU restatement (OpenMP) of the reference's bitvector SpGEMM path and index schedule, not the reference "
            "binary: the reference's Kokkos build cannot be compiled here")


def run_reference(args, rank, world):
    """CPU arm: the restated reference path on the host cores, rank 0 only.
    Every timed step builds the index of the whole graph; warm-up steps build
    the index of a 1e6-base prefix of the same generator (they only start the
    thread pool and the allocator)."""
    if rank != 0:
        return
    from oracle import pyoracle as orc
    a, _ = graph(args.n_backbone, args.seed)
    n_full = a.numRows()
    warm_backbone = min(args.n_backbone, 1_000_000)
    aw, _ = graph(warm_backbone, args.seed)
    for _ in range(args.warmup):
        cpu_build(aw, args.dmin, args.dmax)
    times = []
    entries = None
    for _ in range(args.steps):
        t, idx = cpu_build(a, args.dmin, args.dmax)
        times.append(t)
        entries = int(idx.rowmap[-1])
        del idx
    value = sum(times) / len(times)
    sample = (f"each timed step: one index build [{args.dmin},{args.dmax}] of the whole graph ({n_full} loci, "
              f"{entries // 2} index ranges), no scaling; warm-up steps: a {warm_backbone}-base prefix; "
              + cpu_kind_note())
    line = {
        "impl": "reference", "metric": "index-build s", "value": value, "unit": "s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": config_dict(args, n_full),
        "cpu_baseline": {"value": value, "unit": "s", "cores": orc.threads(), "kind": "port", "sample": sample,
                         "best_s": min(times), "mean_s": value, "per_step_s": [round(t, 3) for t in times]},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def config_dict(args, n_loci):
    return {"workload": "plain index build, synthetic chromosome-scale sequence graph",
            "n_backbone": args.n_backbone, "n_loci": n_loci, "window": [args.dmin, args.dmax],
            "bubbles": "SNP 1/1000, indel 1/5000 (geometric mean 4, cap 50), 0.1% structural (100..2000)",
            "seed": args.seed, "index_types": "uint32 columns, uint64 rowmap",
            "l2": "inputs larger than L2 (A and every intermediate exceed 126 MB)",
            "parallelism": f"{args.gpus} independent graph(s), one per GPU",
            **({"options": list(args.set)} if args.set else {})}


def flush_l2(buf):
    """Reads a buffer larger than L2 (evicts what the last launch left, and
    leaves no dirty lines whose write-back would share the next launch's
    DRAM time)."""
    buf.amax()


# ---- secondary workloads ---------------------------------------------------------

def run_query(args, ctx, stream, d_idx, a, want, npairs=1_000_000, steps=20, warmup=3):
    """Membership queries (dvg_query_batch, k_query) against the resident
    chromosome-scale index: npairs locus pairs, half within the distance
    window, the index (0.8 GB) larger than L2, L2 flushed between launches;
    each launch bracketed by CUDA events.  Answers compared with the oracle's
    restatement of CRSMatrixBase::operator() (crs_matrix.hpp:1197-1218)."""
    import numpy as np
    import torch
    from diverg_b200 import gen
    pairs = gen.query_pairs(a, npairs, 0.5, args.dmin, args.dmax, seed=args.seed + 11)
    d_pairs = torch.from_numpy(pairs.view(np.int32).reshape(-1)).cuda()
    d_out = torch.empty(npairs, dtype=torch.uint8, device="cuda")
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            ctx.query_device(d_idx, d_pairs.data_ptr(), npairs, d_out.data_ptr())
        # the kernel: CUDA-event spans inside the library around each launch
        ctx.set_option("timing", 1)
        ctx.reset_stats()
        ms = []
        for _ in range(steps):
            flush_l2(flush)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ctx.query_device(d_idx, d_pairs.data_ptr(), npairs, d_out.data_ptr())
            e1.record(stream)
            ms.append((e0, e1))
        stream.synchronize()
        st = ctx.stats()
        ctx.set_option("timing", 0)
    call_s = sum(e0.elapsed_time(e1) / 1e3 for e0, e1 in ms) / len(ms)
    mean_s = st["query_ns"] / 1e9 / steps
    got = d_out.cpu().numpy()
    parity = None
    if want is not None:
        from oracle import pyoracle as orc
        parity = bool(np.array_equal(got, orc.query(want, pairs)))
    # e2e: host pairs in, host answers out through the C ABI (one call)
    h_pairs = np.ascontiguousarray(pairs)
    t0 = time.perf_counter()
    for _ in range(3):
        host_ans = ctx.query(d_idx, h_pairs)
    e2e_s = (time.perf_counter() - t0) / 3
    peak, peak_kind = peaks()
    ach = QUERY_ALG_BYTES * npairs / mean_s / 1e9
    # the measured ceiling of random reads: independent 8-byte reads at random
    # addresses of a buffer the size of the index (one sector each), timed by
    # the library; a pair makes at least two (its row pointers, its range)
    idx_bytes = 8 * (d_idx.nrows + 1) + 4 * d_idx.nentries
    rr_peak = ctx.calibrate_random_reads(idx_bytes)
    rr_ach = 2.0 * npairs / mean_s
    return {"metric": "membership queries/s", "value": npairs / mean_s, "unit": "queries/s",
            "higher_is_better": True, "steps": steps, "warmup": warmup,
            "config": {"workload": "membership queries against the resident chromosome-scale index",
                       "pairs": npairs, "in_window_fraction": 0.5, "window": [args.dmin, args.dmax],
                       "l2": "index larger than L2, L2 flushed between launches"},
            "kernel_us": mean_s * 1e6, "ns_per_query": mean_s / npairs * 1e9,
            "call_us": call_s * 1e6,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_kind": peak_kind, "alg_bytes_per_query": QUERY_ALG_BYTES,
                         # a random pair moves whole 32-byte sectors: its row's two
                         # pointers and its range (one sector each at least), its
                         # 8-byte pair and its answer byte
                         "sector_bytes_per_query": QUERY_SECTOR_BYTES,
                         "frac_of_sector_bound": ach / peak * QUERY_SECTOR_BYTES / QUERY_ALG_BYTES,
                         "note": "random rows: every pair touches at least two 32-byte DRAM sectors (rowmap, "
                                 "range), so the 33-byte algorithmic count caps frac at 33/73 of peak",
                         "random_reads": {"achieved": rr_ach, "peak": rr_peak, "unit": "random reads/s",
                                          "frac": rr_ach / rr_peak if rr_peak else None,
                                          "peak_kind": "measured (dvg_calibrate_random_reads over "
                                                       f"{idx_bytes / 1e9:.2f} GB, the index's size)",
                                          "note": "two dependent random reads a pair (row pointers, then "
                                                  "its range) against independent random 8-byte reads"}},
            "e2e": {"value": npairs / e2e_s, "unit": "queries/s", "h2d_bytes_per_step": int(h_pairs.nbytes),
                    "d2h_bytes_per_step": int(npairs), "note": "pageable host buffers, one call"},
            "answers_in_range": int(got.sum()), "parity": parity,
            "e2e_answers_equal": bool(np.array_equal(host_ans, got))}


def range_ops_count(a, b):
    """Work of C = A B on the B side: the B ranges of every B row an A range
    names, summed over A's ranges (numpy on the host)."""
    import numpy as np
    s = a.entries[0::2].astype(np.int64)
    f = a.entries[1::2].astype(np.int64)
    br = np.asarray(b.rowmap, dtype=np.int64)
    return int(((br[f + 1] - br[s]) // 2).sum())


def run_spgemm_micro(args, ctx, stream, rank, steps=None, warmup=None):
    """range_spgemm and range_spadd alone on random banded matrices: n = 2^24,
    band half-width 512, Poisson(4) ranges per row of geometric length
    (mean 32), canonical, fixed seeds.  Device-resident operands, L2 flushed
    between products; each kernel bracketed by CUDA events on the library's
    stream.  Algorithmic bytes are A + B + C of the product (+ nothing for the
    union levels the row kernel builds first: their time is counted, their
    bytes are not)."""
    import torch
    from diverg_b200 import gen
    steps = steps or args.steps
    warmup = warmup or args.warmup
    n = 1 << args.log2_rows
    a = gen.banded(n, 512, 4.0, 32.0, seed=args.seed + 2 * rank)
    b = gen.banded(n, 512, 4.0, 32.0, seed=args.seed + 2 * rank + 1)
    rops = range_ops_count(a, b)
    da, db = ctx.upload(a), ctx.upload(b)
    peak, peak_kind = peaks()
    flush = torch.empty(2 * L2_BYTES // 4, dtype=torch.int32, device="cuda")
    res = {}
    # the on-chip denominator: range operations a second the device sustains
    # for the warp-per-row kernel's inner work (measured by the library)
    variants = (("range_spgemm[automatic]", ctx.spgemm, 0), ("range_spgemm[tile-staged]", ctx.spgemm, 1),
                ("range_spgemm[row+levels]", ctx.spgemm, 2), ("range_spadd", ctx.spadd, 0))
    wanted = {"range_spgemm[" + k + "]" if k != "spadd" else "range_spadd" for k in args.kernels.split(",")}
    unknown = wanted - {v[0] for v in variants}
    if unknown:
        raise SystemExit(f"--kernels: unknown {sorted(unknown)}")
    variants = tuple(v for v in variants if v[0] in wanted)
    rangeop_peak = ctx.calibrate_range_ops() if any(v[0] != "range_spadd" for v in variants) else None
    for name, op, mode in variants:
        ctx.set_option("spgemm_mode", mode)
        for _ in range(warmup):
            op(da, db).free()
        ctx.set_option("timing", 1)
        ctx.reset_stats()
        ranges = 0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush_l2(flush)
            c = op(da, db)
            ranges = c.nentries // 2
            c.free()
        ctx.synchronize()
        st = ctx.stats()
        ctx.set_option("timing", 0)
        if name == "range_spadd":
            kern_ns, lv_ns, alg = st["spadd_ns"] + st["scan_ns"], 0, st["alg_bytes"]
        else:
            kern_ns, lv_ns, alg = st["spgemm_ns"], st["spgemm_levels_ns"], st["spgemm_alg_bytes"]
        kern_s = (kern_ns + lv_ns) / 1e9 / steps
        gbs = alg / steps / kern_s / 1e9
        res[name] = {"kernel_ms": kern_s * 1e3, "product_ms": kern_ns / 1e6 / steps, "levels_ms": lv_ns / 1e6 / steps,
                     "alg_bytes": alg / steps, "achieved_gbs": gbs, "frac": gbs / peak, "output_ranges": ranges,
                     "output_ranges_per_s": ranges / kern_s}
        if name != "range_spadd":
            res[name]["range_ops"] = rops
            res[name]["range_ops_per_s"] = rops / kern_s
            res[name]["onchip"] = {"bound": "range operations", "achieved": rops / kern_s, "peak": rangeop_peak,
                                   "unit": "range ops/s", "frac": rops / kern_s / rangeop_peak,
                                   "peak_kind": "measured (dvg_calibrate_range_ops)"}
    ctx.set_option("spgemm_mode", 0)
    da.free()
    db.free()
    if "range_spgemm[automatic]" not in res:  # a subset without the default kernel: its first, HBM-bound
        name, first = next(iter(res.items()))
        return {"metric": name.split("[")[0] + " HBM GB/s", "value": first["achieved_gbs"], "unit": "GB/s",
                "higher_is_better": True, "dtype": "u32", "data": "synthetic", "steps": steps, "warmup": warmup,
                "config": {"workload": "kernel microbenchmark subset: " + ", ".join(res), "n": n},
                "peak": peak, "peak_kind": peak_kind, "kernels": res,
                "roofline": {"bound": "hbm", "achieved": first["achieved_gbs"], "peak": peak, "unit": "GB/s",
                             "frac": first["frac"]}}
    best = res["range_spgemm[automatic]"]
    return {"metric": "range_spgemm HBM GB/s", "value": best["achieved_gbs"], "unit": "GB/s",
            "higher_is_better": True, "dtype": "u32", "data": "synthetic", "steps": steps, "warmup": warmup,
            "config": {"workload": "kernel microbenchmark: range_spgemm and range_spadd of two random banded "
                                   "matrices", "n": n, "half_width": 512, "ranges_per_row": "Poisson(4)",
                       "range_length": "geometric, mean 32", "seeds": [args.seed, args.seed + 1],
                       "l2": "operands (0.7 GB each) larger than L2, L2 flushed between products"},
            "peak": peak, "peak_kind": peak_kind, "kernels": res,
            "roofline": {"bound": "on-chip", "achieved": best["range_ops_per_s"], "peak": rangeop_peak,
                         "unit": "range ops/s", "frac": best["onchip"]["frac"],
                         "hbm_frac": best["frac"]},
            "note": "value: the automatic kernel choice (warp per row here); range_ops = B ranges named by A's "
                    "ranges, the product's on-chip work; on-chip peak: warps ORing L1-resident ranges into "
                    "shared bitmap windows and gathering runs, measured on this device"}


def cfg3_batch(args, rank, ngraphs):
    """ngraphs graphs of the small-graph generator (bubbles 1/100: 70 % SNP,
    30 % indel of length 1..10), sizes log-normal (median 2e4, sigma 1.0)
    clipped to [1e3, 1e6] bases, windows drawn from {[100,300], [200,500],
    [400,600]}, graph k seeded seed + k."""
    import numpy as np
    from diverg_b200 import gen
    rng = np.random.default_rng(args.seed + 1000 * rank)
    sizes = np.clip(rng.lognormal(np.log(2e4), 1.0, ngraphs), 1e3, 1e6).astype(np.int64)
    wins = [(100, 300), (200, 500), (400, 600)]
    windows = [wins[int(i)] for i in rng.integers(0, 3, ngraphs)]
    graphs = [gen.graph_adjacency(gen.small_graph_spec(int(n), seed=args.seed + 1000 * rank + k))[0]
              for k, n in enumerate(sizes)]
    return graphs, windows


def run_batch(args, ctx, stream, rank, steps=None, warmup=None, oracle_every=20):
    """Batched builds (dvg_batch_distance_index) against back-to-back plain
    builds of the same graphs.  Every graph's batched index is compared entry
    by entry with its plain build, and every oracle_every-th graph with the
    oracle's CPU build."""
    import numpy as np
    import torch
    steps = steps or args.steps
    warmup = warmup or args.warmup
    graphs, windows = cfg3_batch(args, rank, args.graphs)
    dg = [ctx.upload(g) for g in graphs]
    loci = sum(g.numRows() for g in graphs)
    # plain: back-to-back single builds, each bracketed by events
    for k in range(min(50, len(dg))):
        ctx.distance_index(dg[k], *windows[k]).free()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in dg]
    plain = []
    torch.cuda.synchronize()
    for k, (d, w) in enumerate(zip(dg, windows)):
        evs[k][0].record(stream)
        ix = ctx.distance_index(d, *w)
        evs[k][1].record(stream)
        plain.append(ix)
    torch.cuda.synchronize()
    lat_plain = np.array([e0.elapsed_time(e1) for e0, e1 in evs])
    plain_s = evs[0][0].elapsed_time(evs[-1][1]) / 1e3
    plain_host = [ix.download() for ix in plain]
    for ix in plain:
        ix.free()
    # batched: warm-up (the first batch autotunes), then timed batches
    ctx.reset_stats()
    outs = None
    for i in range(warmup):
        outs = ctx.batch_distance_index(dg, windows)
        if i < warmup - 1:
            for o in outs:
                o.free()
    tuned = ctx.stats()["autotune_builds"]
    # parity of the last warm-up batch: every graph against its plain build,
    # every oracle_every-th against the oracle
    same_plain = True
    oracle_checked, oracle_same = 0, True
    from oracle import pyoracle as orc
    for k, o in enumerate(outs):
        h = o.download()
        p = plain_host[k]
        same_plain &= (np.array_equal(h.rowmap, p.rowmap) and np.array_equal(h.entries, p.entries)
                       and h.nnz() == p.nnz())
        if k % oracle_every == 0:
            want = orc.dindex(omat(graphs[k]), *windows[k], algo="hbv")
            oracle_same &= (np.array_equal(h.rowmap, want.rowmap) and np.array_equal(h.entries, want.entries)
                            and h.nnz() == want.nnz)
            oracle_checked += 1
        o.free()
    del plain_host
    ctx.reset_stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(steps):
        outs = ctx.batch_distance_index(dg, windows)
        for o in outs:
            o.free()
    ev1.record(stream)
    torch.cuda.synchronize()
    st = ctx.stats()
    batch_s = ev0.elapsed_time(ev1) / 1e3 / steps
    for d in dg:
        d.free()
    n = len(dg)
    return {"metric": "batched index builds/s", "value": n / batch_s, "unit": "builds/s", "higher_is_better": True,
            "dtype": "u32", "data": "synthetic", "steps": steps, "warmup": warmup,
            "config": {"workload": "batched index builds of mixed-size graphs", "graphs": n, "loci": int(loci),
                       "sizes": "log-normal, median 2e4 bases, sigma 1.0, clipped [1e3, 1e6]",
                       "windows": "uniform over [100,300], [200,500], [400,600]", "seed": args.seed},
            "plain_builds_per_s": n / plain_s, "speedup_vs_plain": plain_s / batch_s,
            "latency_ms": {"batch": batch_s * 1e3, "plain_p50": float(np.percentile(lat_plain, 50)),
                           "plain_p99": float(np.percentile(lat_plain, 99)), "plain_total": plain_s * 1e3},
            "graph_launches_per_batch": st["graph_launches"] / steps,
            "kernel_launches_per_batch": st["kernel_launches"] / steps,
            "autotune_builds": tuned, "parity": {"all_equal_plain": bool(same_plain),
                                                 "oracle_checked": oracle_checked,
                                                 "oracle_equal": bool(oracle_same)}}


def run_adjacency(args, ctx, stream, rank):
    """Adjacency construction (util::range_adjacency_matrix) of the
    chromosome-scale synthetic graph, compacted into nodes, on the device:
    host node lengths and edges in, the range-CRS matrix resident in HBM (the
    step a build starts from).  e2e adds the download of the matrix to pinned
    host buffers.  The CPU baseline is the oracle's single-thread restatement
    of the reference's host construction (adjacency.hpp:170-228 and the
    Basic->Range append, crs_matrix.hpp:197-242) on the same graph."""
    import torch
    from diverg_b200 import gen
    spec = gen.chromosome_graph_spec(args.n_backbone, seed=args.seed + rank)
    lens, edges = gen.graph_nodes(spec)
    nloci = int(lens.sum())
    for _ in range(args.warmup):
        ctx.adjacency_from_graph(lens, edges).free()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ctx.reset_stats()
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(args.steps):
        m = ctx.adjacency_from_graph(lens, edges)
        nentries, nnz = m.nentries, m.nnz
        m.free()
    ev1.record(stream)
    torch.cuda.synchronize()
    st = ctx.stats()
    step_s = ev0.elapsed_time(ev1) / 1e3 / args.steps
    # algorithmic bytes: node lengths and edges in, rows out
    out_bytes = 8 * (nloci + 1) + 4 * nentries
    alg = 4 * len(lens) + 8 * len(edges) + out_bytes
    # e2e: the same plus the matrix into pinned host memory
    o_rowmap = torch.empty(nloci + 1, dtype=torch.int64).pin_memory()
    o_entries = torch.empty(max(1, nentries), dtype=torch.int32).pin_memory()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        m = ctx.adjacency_from_graph(lens, edges)
        m.download_to(o_rowmap.data_ptr(), o_entries.data_ptr())
        m.free()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_s = e0.elapsed_time(e1) / 1e3 / args.steps
    cpu = None
    if not args.no_cpu_baseline and rank == 0:
        from oracle import pyoracle as orc
        t0 = time.perf_counter()
        ref = orc.adjacency(lens, edges)
        cpu_s = time.perf_counter() - t0
        assert len(ref.entries) == nentries
        cpu = {"value": cpu_s, "unit": "s", "cores": 1, "kind": "port",
               "sample": f"the whole graph ({nloci} loci), the oracle's single-thread restatement of the "
                         "reference's host adjacency construction"}
    peak, peak_kind = peaks()
    return {"metric": "adjacency construction s", "value": step_s, "unit": "s", "higher_is_better": False,
            "dtype": "u32", "data": "synthetic",
            "config": {"workload": "range adjacency of the chromosome-scale synthetic graph from its node graph",
                       "n_backbone": args.n_backbone, "nodes": int(len(lens)), "edges": int(len(edges)),
                       "loci": nloci, "seed": args.seed},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(4 * len(lens) + 8 * len(edges)),
                    "d2h_bytes_per_step": int(out_bytes)},
            "roofline": {"bound": "hbm", "achieved": alg / step_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / step_s / 1e9 / peak, "traffic": None, "peak_kind": peak_kind,
                         "note": "whole call (two read-backs size the output), algorithmic bytes over its time"},
            "gpu_launches": st["kernel_launches"] / args.steps, "cpu_baseline": cpu,
            "index": {"entries": int(nentries), "nnz": int(nnz)}}


def apply_options(ctx, pairs):
    for kv in pairs:
        key, _, value = kv.partition("=")
        ctx.set_option(key.strip(), int(value))


def secondary(args, ctx, stream, local, d_idx, a, want):
    """The secondary workloads after the headline (N = 1), each with its own
    clock samples and its own step counts (stated in its entry)."""
    from diverg_b200 import serving
    out = {}
    jobs = [("query", lambda: run_query(args, ctx, stream, d_idx, a, want)),
            ("spgemm", lambda: run_spgemm_micro(args, ctx, stream, 0, steps=5, warmup=3)),
            ("batch", lambda: run_batch(args, ctx, stream, 0, steps=5, warmup=3)),
            ("serve", lambda: serving.bench_line(args, ctx, 0, requests=600))]
    for name, job in jobs:
        try:
            with ClockSampler([local]) as clocks:
                r = job()
            r["clocks"] = clocks.summary()
        except Exception as e:  # a secondary failure must not hide the headline
            r = {"error": f"{type(e).__name__}: {e}"}
        out[name] = r
    return out


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload != "build":
        run_other(args, rank, world, local)
        return

    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    from diverg_b200.runtime import Context

    a, gstats = graph(args.n_backbone, args.seed + rank)
    n_loci = a.numRows()
    ctx = Context(local)
    apply_options(ctx, args.set)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    d_a = ctx.upload(a)

    # warm-up; the first warm-up build's index is kept on the host for the
    # parity check (freed on the device, so the timed builds find the
    # allocator as every later build does)
    first = None
    for i in range(args.warmup):
        d_idx = ctx.distance_index(d_a, args.dmin, args.dmax)
        idx_rows, idx_entries, idx_nnz = d_idx.nrows, d_idx.nentries, d_idx.nnz
        if i == 0 and rank == 0 and world == 1 and not args.no_cpu_baseline:
            first = d_idx.download()
        d_idx.free()

    # ---- timed: device-resident input -------------------------------------
    ctx.reset_stats()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler([local] if world == 1 else list(range(world))) as clocks:
        barrier()
        torch.cuda.synchronize()
        ev0.record(stream)
        wall = []
        for _ in range(args.steps):
            w0 = time.perf_counter()
            idx = ctx.distance_index(d_a, args.dmin, args.dmax)
            idx.free()
            wall.append((time.perf_counter() - w0) * 1e3)
        ev1.record(stream)
        torch.cuda.synchronize()
        barrier()
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    st_timed = ctx.stats()
    launches = st_timed["kernel_launches"]
    sec_per_build = ms_total / 1e3 / args.steps

    # ---- the same builds again with per-kernel event spans (roofline) ------
    ctx.set_option("timing", 1)
    ctx.reset_stats()
    for _ in range(args.steps):
        idx = ctx.distance_index(d_a, args.dmin, args.dmax)
        idx.free()
    ctx.synchronize()
    st = ctx.stats()
    ctx.set_option("timing", 0)

    # ---- e2e: host buffers through the C ABI ---------------------------------
    e2e = None
    if not args.no_e2e:
        h_rowmap = torch.from_numpy(a.rowmap.astype(np.uint64).view(np.int64)).pin_memory()
        h_entries = torch.from_numpy(a.entries.view(np.int32)).pin_memory()
        o_rowmap = torch.empty(idx_rows + 1, dtype=torch.int64).pin_memory()
        o_entries = torch.empty(max(1, idx_entries), dtype=torch.int32).pin_memory()
        h2d = h_rowmap.numel() * 8 + h_entries.numel() * 4
        d2h = (idx_rows + 1) * 8 + idx_entries * 4
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(args.steps):
            da2 = ctx.upload_arrays(n_loci, n_loci, h_rowmap.data_ptr(), h_entries.data_ptr(), a.nnz())
            ix = ctx.distance_index(da2, args.dmin, args.dmax)
            ix.download_to(o_rowmap.data_ptr(), o_entries.data_ptr())
            ix.free()
            da2.free()
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        e2e_s = max_over_ranks(e0.elapsed_time(e1)) / 1e3 / args.steps
        e2e = {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)}
        del h_rowmap, h_entries, o_rowmap, o_entries

    # ---- roofline of the range-SpGEMM kernel ------------------------------
    peak, peak_kind = peaks()
    spgemm_ns = st["spgemm_ns"]
    spgemm_calls = max(1, st["spgemm_calls"])
    per_product_bytes = st["spgemm_alg_bytes"] / spgemm_calls
    per_product_s = spgemm_ns / 1e9 / spgemm_calls
    achieved = per_product_bytes / per_product_s / 1e9 if per_product_s > 0 else None
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": (achieved / peak) if achieved else None,
                "traffic": ROWMODE_TRAFFIC_BYTES_PER_ROW * n_loci,
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                  "the row kernel's capture on the 1e7-base graph (profiles/), scaled by rows",
                "peak_kind": peak_kind,
                "kernel": "k_spgemm_rowmode (single-pass range SpGEMM: counts, chunk look-back, runs)",
                "alg_bytes_per_product": per_product_bytes, "products_per_build": st["spgemm_calls"] / args.steps}

    # ---- CPU baseline on the whole graph; its index is the parity oracle ---
    cpu, want, parity, parity_detail = None, None, None, None
    if first is not None:
        t_cpu, want = cpu_build(a, args.dmin, args.dmax)
        from oracle import pyoracle as orc
        cpu = {"value": t_cpu, "unit": "s", "cores": orc.threads(), "kind": "port",
               "sample": f"one index build [{args.dmin},{args.dmax}] of the whole graph ({n_loci} loci), no "
                         f"scaling; " + cpu_kind_note()}
        got = first
        same_rowmap = bool(np.array_equal(got.rowmap.astype(np.uint64), want.rowmap))
        same_entries = bool(np.array_equal(got.entries, want.entries))
        same_nnz = got.nnz() == int(want.nnz)
        parity = same_rowmap and same_entries and same_nnz
        parity_detail = {"oracle": "the CPU baseline's index (reference schedule, bitvector SpGEMM)",
                         "gpu_build": "the first warm-up build", "rowmap_equal": same_rowmap,
                         "entries_equal": same_entries, "nnz_equal": same_nnz,
                         "rows": int(got.numRows()), "entries": int(got.entries.size), "nnz": int(got.nnz())}
        del got, first

    sec = None
    if world == 1 and not args.no_secondary:
        d_idx = ctx.distance_index(d_a, args.dmin, args.dmax)  # resident index for the queries
        sec = secondary(args, ctx, stream, local, d_idx, a, want)
        d_idx.free()
    del want

    if rank == 0:
        steps = args.steps
        line = {
            "metric": "index-build s", "value": sec_per_build, "unit": "s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": sec_per_build * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic",
            "config": config_dict(args, n_loci),
            "e2e": e2e,
            "gpu_launches": launches,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "parity": parity,
            "parity_detail": parity_detail,
            "clocks": clocks.summary(),
            "build": {"index_rows": idx_rows, "index_ranges": idx_entries // 2, "index_nnz": idx_nnz,
                      "graph": gstats, "spgemm_per_build": st["spgemm_calls"] / steps,
                      "alg_gb_per_build": st["alg_bytes"] / steps / 1e9,
                      "build_gbs": st["alg_bytes"] / steps / 1e9 / sec_per_build,
                      "kernel_ms_per_build": {
                          "spgemm": st["spgemm_ns"] / 1e6 / steps,
                          "spgemm_levels": st["spgemm_levels_ns"] / 1e6 / steps,
                          "scan": st["scan_ns"] / 1e6 / steps, "spadd": st["spadd_ns"] / 1e6 / steps},
                      "host_syncs_per_build": st["host_syncs"] / steps,
                      # host side of the timed builds: where the GPU could idle
                      "host_ms_per_build": {
                          "wall_per_step": [round(w, 2) for w in wall],
                          "prepare": st_timed["host_prepare_ns"] / 1e6 / steps,
                          "meminfo": st_timed["host_meminfo_ns"] / 1e6 / steps,
                          "launch": st_timed["host_launch_ns"] / 1e6 / steps,
                          "sync_wait": st_timed["host_sync_ns"] / 1e6 / steps}},
            "secondary": sec,
        }
        print(json.dumps(line), flush=True)

    d_a.free()
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_other(args, rank, world, local):
    """The secondary workloads on their own: one replica per rank, rank 0
    prints its line."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from diverg_b200.runtime import Context
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    ctx = Context(local)
    apply_options(ctx, args.set)
    stream = torch.cuda.Stream()
    ctx.set_stream(stream.cuda_stream)
    with ClockSampler([local]) as clocks:
        if args.workload == "spgemm":
            line = run_spgemm_micro(args, ctx, stream, rank)
        elif args.workload == "batch":
            line = run_batch(args, ctx, stream, rank)
        elif args.workload == "adjacency":
            line = run_adjacency(args, ctx, stream, rank)
        elif args.workload == "query":
            a, _ = graph(args.n_backbone, args.seed + rank)
            d_a = ctx.upload(a)
            d_idx = ctx.distance_index(d_a, args.dmin, args.dmax)
            want = None
            if not args.no_cpu_baseline:
                _, want = cpu_build(a, args.dmin, args.dmax)
            line = run_query(args, ctx, stream, d_idx, a, want, steps=args.steps, warmup=args.warmup)
            d_idx.free()
            d_a.free()
        else:
            from diverg_b200 import serving
            line = serving.bench_line(args, ctx, rank)
    line.update({"n_gpus": world, "steps": line.get("steps", args.steps),
                 "warmup": line.get("warmup", args.warmup), "clocks": clocks.summary(),
                 "scaling": "weak", "vs_baseline": None})
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
