"""A sequence graph read from GFA 1 or GFA 2 text, ready for
Context.adjacency_from_graph: node lengths in rank order and the forward
edges as 1-based (from rank, to rank) pairs.

The reference loads graphs with gum (gum::util::load_gfa over GFAKluge,
benchmark/src/rcrs_benchmark.hpp:292-376 in cartoonist/diverg) and orders the
nodes ("native": the file's order; "topological"; others); gum is absent
here, so this reader follows the GFA specifications, as include/diverg/gfa.hpp
does for C++: segments (GFA 1 ``S name seq [LN:i:len]``, GFA 2
``S sid slen seq``) are the nodes, links (GFA 1 ``L from + to + overlap``) and
edges (GFA 2 ``E eid sid1+ sid2+ ...``) the forward edges.  "native" ranks the
nodes in file order; "topological" by Kahn's algorithm taking the lowest
file position first, with the nodes of cycles ranked after in file order.
Edges between opposite strands are rejected."""
import heapq

import numpy as np


class GFAError(ValueError):
    pass


def _is_gfa2_segment(f):
    return len(f) >= 4 and f[2].isdigit() and ":" not in f[3]


def parse(text, ordering="native"):
    """(node_len uint32[n], edges uint32[m, 2] of 1-based ranks, names in rank order)."""
    if ordering not in ("native", "topological"):
        raise GFAError(f"unknown ordering {ordering!r}")
    names, lens, links, index = [], [], [], {}
    for line in text.splitlines():
        f = line.rstrip("\r").split("\t")
        if not f or not f[0]:
            continue
        if f[0] == "S":
            if len(f) < 3:
                raise GFAError("short S line")
            if _is_gfa2_segment(f):
                length = int(f[2])
            elif f[2] != "*":
                length = len(f[2])
            else:
                length = 0
                for t in f[3:]:
                    if t.startswith("LN:i:"):
                        length = int(t[5:])
            if f[1] in index:
                raise GFAError(f"segment {f[1]} defined twice")
            index[f[1]] = len(names)
            names.append(f[1])
            lens.append(length)
        elif f[0] == "L":
            if len(f) < 5:
                raise GFAError("short L line")
            if f[2] != "+" or f[4] != "+":
                raise GFAError("reverse-strand edges are not supported")
            links.append((f[1], f[3]))
        elif f[0] == "E":
            if len(f) < 4:
                raise GFAError("short E line")
            ends = []
            for s in (f[2], f[3]):
                if not s or s[-1] not in "+-":
                    raise GFAError(f"bad segment reference {s}")
                if s[-1] == "-":
                    raise GFAError("reverse-strand edges are not supported")
                ends.append(s[:-1])
            links.append(tuple(ends))
    n = len(names)
    succ = [[] for _ in range(n)]
    for a, b in links:
        if a not in index or b not in index:
            raise GFAError("edge to an unknown segment")
        succ[index[a]].append(index[b])
    if ordering == "native":
        order = list(range(n))
    else:
        indeg = [0] * n
        for k in range(n):
            for t in succ[k]:
                indeg[t] += 1
        ready = [k for k in range(n) if indeg[k] == 0]
        heapq.heapify(ready)
        order, done = [], [False] * n
        while ready:
            k = heapq.heappop(ready)
            order.append(k)
            done[k] = True
            for t in succ[k]:
                indeg[t] -= 1
                if indeg[t] == 0:
                    heapq.heappush(ready, t)
        order += [k for k in range(n) if not done[k]]
    rank = np.empty(n, dtype=np.int64)
    rank[order] = np.arange(1, n + 1)
    node_len = np.array([lens[k] for k in order], dtype=np.uint32)
    edges = [(rank[k], rank[t]) for k in order for t in succ[k]]
    edges = np.array(edges, dtype=np.uint32).reshape(-1, 2)
    return node_len, edges, [names[k] for k in order]


def load(path, ordering="native"):
    with open(path) as fh:
        return parse(fh.read(), ordering)
