"""Generate the golden fixtures in tests/golden/golden.npz.

Each case is a small ECLgraph (nindex, nlist, eweight) built here with numpy
from a fixed seed, plus the outputs of the REFERENCE ITSELF on it: the inMST
array of the reference cpuMST (ECL-MST/ECL_MST.cu:82-124) and the threshold
choice of the reference main (:408,:432-444), both taken from
oracle/_ref/libecl_ref.so, which oracle/Makefile compiles from the unmodified
reference source. Run from the repository root after `make -C oracle`:

    python tests/golden/make_golden.py

The cases cover what the reference path has to get right: ties broken by the
edge index, parallel edges, self-loops, isolated vertices and many
components, asymmetric CSR (one direction missing), a single vertex, an empty
edge set, hubs whose rows cross the 128-entry chunk boundary, long hook
chains (paths with monotone weights), unsorted rows, extreme weights, and
graphs dense enough (edges/nodes >= 4) to take the filtered two-phase path.
"""
import ctypes
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "golden.npz")


def csr_from_pairs(n, pairs, weights, symmetric=True, sort_rows=True, rng=None):
    """pairs: list of (u, v); weights parallel. Symmetric adds (v, u) with the same weight."""
    src, dst, w = [], [], []
    for (u, v), x in zip(pairs, weights):
        src.append(u); dst.append(v); w.append(x)
        if symmetric:
            src.append(v); dst.append(u); w.append(x)
    src = np.array(src, np.int64); dst = np.array(dst, np.int64); w = np.array(w, np.int64)
    if sort_rows:
        order = np.lexsort((dst, src))
    else:
        order = np.argsort(src, kind="stable")
        if rng is not None:  # shuffle within rows
            key = rng.random(len(src))
            order = np.lexsort((key, src))
    src, dst, w = src[order], dst[order], w[order]
    nindex = np.zeros(n + 1, np.int32)
    np.add.at(nindex, src + 1, 1)
    nindex = np.cumsum(nindex).astype(np.int32)
    return nindex, dst.astype(np.int32), w.astype(np.int32)


def cases():
    rng = np.random.default_rng(20231112)
    out = []

    def add(name, n, pairs, weights, **kw):
        out.append((name,) + csr_from_pairs(n, pairs, weights, **kw))

    add("single_vertex", 1, [], [])
    add("one_edge", 2, [(0, 1)], [7])
    add("triangle_ties", 3, [(0, 1), (1, 2), (0, 2)], [5, 5, 5])
    add("parallel_edges", 3, [(0, 1), (0, 1), (1, 2), (1, 2), (0, 2)], [4, 4, 9, 3, 3])
    add("self_loops", 4, [(0, 0), (0, 1), (1, 1), (1, 2), (2, 3), (3, 3)], [1, 5, 1, 6, 2, 1])
    add("isolated_and_components", 12, [(0, 1), (2, 3), (3, 4), (2, 4), (7, 8), (9, 10)],
        [3, 1, 2, 2, 8, 8])
    # asymmetric: only one direction stored for some edges
    out.append(("asymmetric",) + csr_from_pairs(6, [(0, 1), (2, 1), (3, 4), (5, 4), (0, 5), (2, 3)],
                                                  [2, 3, 4, 1, 9, 9], symmetric=False))
    # hub: vertex 0 connected to 300 others, crossing chunk boundaries
    hub_pairs = [(0, i) for i in range(1, 301)] + [(i, i + 1) for i in range(1, 300)]
    add("hub_300", 301, hub_pairs, list(rng.integers(1, 50, len(hub_pairs))))
    # hub whose row starts at an odd offset, not vertex 0
    hub2 = [(i, i + 1) for i in range(0, 9)] + [(5, j) for j in range(10, 400)]
    add("hub_offset", 400, hub2, list(rng.integers(1, 1000, len(hub2))))
    # long chains: monotone weights along a path
    P = 3000
    add("path_increasing", P, [(i, i + 1) for i in range(P - 1)], list(range(1, P)))
    add("path_decreasing", P, [(i, i + 1) for i in range(P - 1)], list(range(P - 1, 0, -1)))
    add("path_equal", P, [(i, i + 1) for i in range(P - 1)], [1] * (P - 1))
    # complete graph
    K = 24
    kp = [(i, j) for i in range(K) for j in range(i + 1, K)]
    add("complete_24", K, kp, list(rng.integers(1, 10**6, len(kp))))
    add("complete_24_ties", K, kp, list(rng.integers(1, 3, len(kp))))
    # random graphs with heavy ties (filtered: avg degree >= 4)
    for s in range(4):
        n = int(rng.integers(50, 400))
        m = int(n * rng.integers(3, 12))
        u = rng.integers(0, n, m); v = rng.integers(0, n, m)
        wmax = [2, 5, 1000, 2**31 - 1][s]
        w = rng.integers(0 if s == 3 else 1, wmax, m, endpoint=True)
        add(f"random_ties_{s}", n, list(zip(u.tolist(), v.tolist())), w.tolist())
    # unsorted rows
    n = 200
    u = rng.integers(0, n, 1500); v = rng.integers(0, n, 1500)
    out.append(("unsorted_rows",) + csr_from_pairs(n, list(zip(u.tolist(), v.tolist())),
                                                     rng.integers(1, 100, 1500).tolist(),
                                                     sort_rows=False, rng=rng))
    # extreme weights: 0, 1, INT_MAX
    n = 64
    pairs = [(i, (i * 7 + 3) % n) for i in range(n)] + [(i, (i * 13 + 5) % n) for i in range(n)]
    ext = rng.choice(np.array([0, 1, 2**31 - 1, 2**31 - 2], np.int64), len(pairs))
    add("extreme_weights", n, pairs, ext.tolist())
    # grid with all-equal weights (tie-breaking by index only)
    R = C = 60
    gp = []
    for r in range(R):
        for c in range(C):
            i = r * C + c
            if c + 1 < C: gp.append((i, i + 1))
            if r + 1 < R: gp.append((i, i + C))
    add("grid_equal", R * C, gp, [1] * len(gp))
    add("grid_random", R * C, gp, rng.integers(1, 10**6, len(gp)).tolist())
    # dense enough for the filter, bigger: exercises several Boruvka rounds
    n = 3000
    m = n * 10
    u = rng.integers(0, n, m); v = rng.integers(0, n, m)
    add("random_dense_3000", n, list(zip(u.tolist(), v.tolist())), rng.integers(1, 2**24, m).tolist())
    # star forest: many small components
    sp = []
    for c in range(100):
        base = c * 10
        sp += [(base, base + k) for k in range(1, 10)]
    add("star_forest", 1000 + 17, sp, rng.integers(1, 20, len(sp)).tolist())
    return out


def main():
    lib_path = os.path.join(ROOT, "oracle", "_ref", "libecl_ref.so")
    if not os.path.exists(lib_path):
        sys.exit("build the reference first: make -C oracle")
    ref = ctypes.CDLL(lib_path)
    P = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    blob = {}
    names = []
    for name, nindex, nlist, w in cases():
        n, m = len(nindex) - 1, len(nlist)
        inmst = np.zeros(max(m, 1), np.uint8)
        ref.ref_cpu_mst(n, m, P(nindex), P(nlist), P(w), P(inmst))
        f, t = ctypes.c_int(), ctypes.c_int()
        if m > 0:
            ref.ref_threshold(n, m, P(w), ctypes.byref(f), ctypes.byref(t))
        else:
            f.value, t.value = 0, 2**31 - 1
        blob[f"{name}/nindex"] = nindex
        blob[f"{name}/nlist"] = nlist
        blob[f"{name}/eweight"] = w
        blob[f"{name}/inMST"] = inmst[:m]
        blob[f"{name}/threshold"] = np.array([t.value, f.value], np.int32)
        names.append(name)
        print(f"{name:28s} n={n:6d} m={m:7d} forest={int(inmst[:m].sum()):6d} "
              f"filter={f.value} thr={t.value}")
    blob["names"] = np.array(names)
    np.savez_compressed(OUT, **blob)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
