"""The request loop (dvg_server_*): index builds and query batches submitted as
they arrive, indices resident in HBM, builds admitted against a memory budget
and batched, query batches overlapping the builds on the device.

`Server` wraps the C ABI; `bench_line` drives it with a Poisson stream of
mixed requests (20 % builds of graphs of 1e4..1e6 bases, 80 % query batches of
1e5..1e6 locus pairs, half of them within the distance window) and reports
throughput with p50 / p99 latencies per arrival rate.
"""
import ctypes
import time

import numpy as np

from . import _native as N
from .crs_matrix import CRSMatrix

BUILD, QUERY = 1, 2


class Server:
    """A dvg_server on one device.  Arrays handed to a request are kept alive
    here until its completion has been polled."""

    def __init__(self, device=0, hbm_budget_bytes=0, max_batch_builds=0, max_inflight_queries=0, build_workers=0):
        cfg = N.ServerConfig(device, int(hbm_budget_bytes), int(max_batch_builds), int(max_inflight_queries),
                             int(build_workers))
        h = ctypes.c_void_p()
        N.check(N.lib().dvg_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._h = h
        self._keep = {}

    def close(self):
        if self._h is not None:
            N.check(N.lib().dvg_server_destroy(self._h))
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit_build(self, m: CRSMatrix, dmin, dmax):
        rowmap = np.ascontiguousarray(m.rowmap, dtype=np.uint64)
        entries = np.ascontiguousarray(m.entries, dtype=np.uint32)
        rid = ctypes.c_uint64()
        N.check(N.lib().dvg_server_submit_build(self._h, m.numRows(), N.ptr(rowmap), N.ptr(entries), dmin, dmax,
                                                ctypes.byref(rid)))
        self._keep[rid.value] = (rowmap, entries)
        return rid.value

    def submit_query(self, index, pairs, answers, npairs=None):
        """pairs: uint32 array (npairs x 2) or a pinned torch tensor; answers:
        uint8 array or pinned tensor of at least npairs elements."""
        p_ptr, n = _buffer(pairs, 8)
        a_ptr, _ = _buffer(answers, 1)
        n = n if npairs is None else int(npairs)
        rid = ctypes.c_uint64()
        N.check(N.lib().dvg_server_submit_query(self._h, index, ctypes.c_void_p(p_ptr), n, ctypes.c_void_p(a_ptr),
                                                ctypes.byref(rid)))
        self._keep[rid.value] = (pairs, answers)
        return rid.value

    def poll(self, max_items=256, wait_ms=0):
        buf = (N.Completion * max_items)()
        n = ctypes.c_uint32()
        N.check(N.lib().dvg_server_poll(self._h, buf, max_items, ctypes.byref(n), wait_ms))
        out = []
        for k in range(n.value):
            c = buf[k]
            self._keep.pop(c.request, None)
            out.append({f: getattr(c, f) for f, _ in N.Completion._fields_})
        return out

    def wait(self, ids, timeout_s=600.0):
        """Polls until every request in `ids` completed; returns their completions."""
        want, got = set(ids), {}
        t_end = time.time() + timeout_s
        while want - set(got):
            if time.time() > t_end:
                raise TimeoutError(f"{len(want - set(got))} requests still pending")
            for c in self.poll(wait_ms=20):
                got[c["request"]] = c
        return [got[i] for i in ids]

    def download(self, index) -> CRSMatrix:
        nr, ne, nz = ctypes.c_uint32(), ctypes.c_uint64(), ctypes.c_uint64()
        N.check(N.lib().dvg_server_index_info(self._h, index, ctypes.byref(nr), ctypes.byref(ne), ctypes.byref(nz)))
        rowmap = np.empty(nr.value + 1, np.uint64)
        entries = np.empty(ne.value, np.uint32)
        N.check(N.lib().dvg_server_download(self._h, index, N.ptr(rowmap), N.ptr(entries)))
        return CRSMatrix(nr.value, entries, rowmap, nz.value)

    def release(self, index):
        N.check(N.lib().dvg_server_release(self._h, index))

    def stats(self):
        s = N.ServerStats()
        N.check(N.lib().dvg_server_get_stats(self._h, ctypes.byref(s)))
        return s.as_dict()


def _buffer(x, itemsize):
    """(address, elements / (itemsize-sized) units) of a numpy array or tensor."""
    if hasattr(x, "data_ptr"):
        return x.data_ptr(), x.numel() * x.element_size() // itemsize
    a = np.asarray(x)
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("buffer must be contiguous")
    return a.ctypes.data, a.nbytes // itemsize


# ---- the mixed-request benchmark --------------------------------------------------

def _percentiles(v):
    v = np.asarray(v, dtype=np.float64)
    if v.size == 0:
        return {"p50": None, "p99": None, "n": 0}
    return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99)), "n": int(v.size)}


def run_stream(server, graphs, pair_pool, answer_pool, rate, nreq, seed, window=(200, 500)):
    """Submits nreq requests at Poisson arrival times (rate per second): 20 %
    builds of graphs[k % len(graphs)], 80 % query batches against a uniformly
    drawn earlier build.  Returns latencies (ms) per kind and the throughput."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, nreq)
    gaps *= (nreq / rate) / gaps.sum()  # the stream's mean rate is the nominal one
    kinds = rng.random(nreq) < 0.2
    sizes = rng.integers(100_000, 1_000_001, nreq)
    built = []          # (build id, graph index)
    free_answers = list(range(len(answer_pool)))
    owner = {}          # query request -> answer buffer slot
    done = {}
    t0 = time.perf_counter()
    t_next = t0
    submitted = []

    def drain(wait_ms=0):
        for c in server.poll(wait_ms=wait_ms):
            done[c["request"]] = c
            slot = owner.pop(c["request"], None)
            if slot is not None:
                free_answers.append(slot)

    for k in range(nreq):
        t_next += gaps[k]
        while True:
            drain()
            now = time.perf_counter()
            if now >= t_next:
                break
            time.sleep(min(t_next - now, 0.0005))
        if kinds[k] or not built:
            gi = len(built) % len(graphs)
            rid = server.submit_build(graphs[gi], *window)
            built.append((rid, gi))
            submitted.append((rid, BUILD))
        else:
            while not free_answers:
                drain(wait_ms=1)
            rid_b, gi = built[int(rng.integers(0, len(built)))]
            n = int(sizes[k])
            slot = free_answers.pop()
            rid = server.submit_query(rid_b, pair_pool[gi], answer_pool[slot], npairs=n)
            owner[rid] = slot
            submitted.append((rid, QUERY))
    while len(done) < len(submitted):
        drain(wait_ms=20)
    t_end = time.perf_counter()
    lat = {BUILD: [], QUERY: []}
    failed = 0
    last_done = 0
    first_submit = last_submit = None
    for rid, kind in submitted:
        c = done[rid]
        failed += c["status"] != N.OK
        lat[kind].append((c["done_ns"] - c["submit_ns"]) / 1e6)
        last_done = max(last_done, c["done_ns"])
        first_submit = c["submit_ns"] if first_submit is None else min(first_submit, c["submit_ns"])
        last_submit = c["submit_ns"] if last_submit is None else max(last_submit, c["submit_ns"])
    span_s = (last_done - first_submit) / 1e9
    # the rate actually offered: the submitting loop can fall behind the
    # arrival times
    offered = (nreq - 1) / max((last_submit - first_submit) / 1e9, 1e-9)
    return {"rate": rate, "offered": offered, "requests": nreq, "failed": failed, "throughput": nreq / span_s,
            "wall_s": t_end - t0, "build_latency_ms": _percentiles(lat[BUILD]),
            "query_latency_ms": _percentiles(lat[QUERY]),
            "all_latency_ms": _percentiles(lat[BUILD] + lat[QUERY]), "builds": [b for b, _ in built]}


def served_ok(r):
    """A rate is served when nothing failed and the requests completed at
    >= 95 % of the rate they were offered at (and of the nominal rate)."""
    return (r["failed"] == 0 and r["throughput"] >= 0.95 * r["offered"]
            and r["offered"] >= 0.9 * r["rate"])


def bench_line(args, ctx, rank, requests=None, max_rate=51200.0):
    """The serving benchmark: graphs of 1e4..1e6 bases (log-uniform) from the
    small-graph generator, window [200, 500], query batches of 1e5..1e6 pairs
    (half within the window), HBM budget 150 GB, Poisson arrivals.  Without a
    fixed rate the sweep doubles the arrival rate from 200/s until the served
    throughput falls below 95 % of the offered rate (or a request fails): the
    knee is the highest rate still served at >= 95 % of the rate actually
    offered (the submitting loop can fall behind), and the first rate past
    it is reported beside it."""
    import torch
    from . import gen
    nreq = int(requests or args.requests)
    rng = np.random.default_rng(args.seed + 7 * rank)
    ngraphs = 48
    sizes = np.exp(rng.uniform(np.log(1e4), np.log(1e6), ngraphs)).astype(np.int64)
    graphs = [gen.graph_adjacency(gen.small_graph_spec(int(n), seed=args.seed + 7 * rank + k))[0]
              for k, n in enumerate(sizes)]
    pair_pool = []
    for k, g in enumerate(graphs):
        p = gen.query_pairs(g, 1_000_000, 0.5, 200, 500, seed=args.seed + k)
        pair_pool.append(torch.from_numpy(p.view(np.int32)).pin_memory())
    answer_pool = [torch.empty(1_000_000, dtype=torch.uint8).pin_memory() for _ in range(64)]
    sweep = []
    saturated = None
    with Server(device=ctx.device, hbm_budget_bytes=150 * 10**9, max_inflight_queries=8) as srv:
        warm = [srv.submit_build(g, 200, 500) for g in graphs[:8]]
        srv.wait(warm)
        rate, i = (args.rate if args.rate > 0 else 200.0), 0
        while True:
            r = run_stream(srv, graphs, pair_pool, answer_pool, rate, nreq, args.seed + 100 + i)
            for b in r.pop("builds"):
                srv.release(b)
            sweep.append(r)
            ok = served_ok(r)
            if args.rate > 0:
                break
            if not ok:
                saturated = r
                break
            if rate * 2 > max_rate:
                break
            rate *= 2
            i += 1
        st = srv.stats()
    served = [r for r in sweep if served_ok(r)]
    knee = max(served, key=lambda r: r["rate"]) if served else min(sweep, key=lambda r: r["rate"])
    return {"metric": "served requests/s", "value": knee["throughput"], "unit": "requests/s",
            "higher_is_better": True, "dtype": "u32", "data": "synthetic",
            "config": {"workload": "serving loop over a mixed Poisson-arrival stream", "builds": "20 %, graphs of "
                       "1e4..1e6 bases (log-uniform), window [200,500]", "queries": "80 %, batches of 1e5..1e6 "
                       "pairs, half within the window", "hbm_budget_gb": 150, "requests_per_rate": nreq,
                       "seed": args.seed},
            "knee_rate": knee["rate"], "latency_ms_at_knee": {"build": knee["build_latency_ms"],
                                                              "query": knee["query_latency_ms"],
                                                              "all": knee["all_latency_ms"]},
            "saturated_at": None if saturated is None else {"rate": saturated["rate"],
                                                            "throughput": saturated["throughput"],
                                                            "failed": saturated["failed"]},
            "knee_measured": saturated is not None,
            "sweep": sweep, "server": st}
