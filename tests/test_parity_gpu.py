"""Parity of the CUDA path (through the C ABI) with the oracle and with the
reference itself rebuilt for sm_100a. Bit-exact inMST and equal uint64 forest
weight on every input: integer work, so the tolerance is zero."""
import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O

pytestmark = pytest.mark.gpu

MODES = [
    dict(),
    dict(mode=E.THRESH_NONE),
    dict(mode=E.THRESH_QUANTILE, quantile=0.05),
    dict(mode=E.THRESH_QUANTILE, quantile=0.5),
    dict(mode=E.THRESH_QUANTILE, quantile=0.95),
    dict(degree_split=1),
    dict(degree_split=4),
    dict(degree_split=1 << 20),
    dict(small_tail=-1),
    dict(small_tail=1 << 30),
    dict(round_min_tiles=-1),
    dict(round_min_tiles=16, small_tail=-1),
    dict(ctas_per_sm=1),
    dict(ctas_per_sm=1, round_min_tiles=-1, small_tail=-1),
    dict(mode=E.THRESH_QUANTILE, quantile=0.3, degree_split=2, small_tail=-1),
    # ablation switches: each turns a technique off; the answer must not change
    dict(flags=E.FLAG_NO_GUARDS),
    dict(flags=E.FLAG_NO_WARP_COOP),
    dict(flags=E.FLAG_DEDUP),
    dict(flags=E.FLAG_NO_FIND_CACHE),
    dict(flags=E.FLAG_L2_PERSIST),
    # the reference's later deoptimization steps, alone and stacked
    dict(flags=E.FLAG_NO_IMPLICIT_COMPRESSION),
    dict(flags=E.FLAG_NO_TUPLES),
    dict(flags=E.FLAG_NO_DATA_DRIVEN),
    dict(flags=E.FLAG_NO_EDGE_BASED),
    dict(flags=E.FLAG_NO_TUPLES | E.FLAG_NO_DATA_DRIVEN | E.FLAG_NO_FIND_CACHE),
    dict(flags=E.FLAG_NO_GUARDS | E.FLAG_NO_WARP_COOP | E.FLAG_NO_IMPLICIT_COMPRESSION | E.FLAG_NO_TUPLES
         | E.FLAG_NO_DATA_DRIVEN | E.FLAG_NO_EDGE_BASED, mode=E.THRESH_NONE),
    dict(flags=E.FLAG_L2_PERSIST | E.FLAG_NO_GRAPH, mode=E.THRESH_QUANTILE, quantile=0.2),
    dict(flags=E.FLAG_NO_GUARDS | E.FLAG_NO_WARP_COOP | E.FLAG_DEDUP | E.FLAG_NO_FIND_CACHE
         | E.FLAG_NO_SMALL_TAIL, mode=E.THRESH_NONE),
]


@pytest.fixture(scope="module")
def ctx():
    c = E.Context(1 << 22, 1 << 26)
    yield c
    c.close()


def _graph(c):
    return E.Graph(c["nindex"], c["nlist"], c["eweight"])


def test_golden_one_shot_entry_point(golden):
    for name, c in golden.items():
        got, st = E.mst(_graph(c))
        assert np.array_equal(got, c["inMST"]), name


@pytest.mark.parametrize("kw", MODES, ids=[str(k) for k in MODES])
def test_golden_every_schedule(ctx, golden, kw):
    opts = E.make_opts(**kw)
    for name, c in golden.items():
        g = _graph(c)
        got, st = ctx.run_host(g, opts)
        assert st["status"] == 0, name
        assert np.array_equal(got, c["inMST"]), (name, kw)
        assert st["forest_weight"] == int(c["eweight"][c["inMST"].astype(bool)].astype(np.int64).sum()) % 2**64


def test_golden_explicit_thresholds(ctx, golden):
    rng = np.random.default_rng(3)
    for name, c in golden.items():
        if len(c["nlist"]) == 0:
            continue
        for t in list(rng.choice(c["eweight"], 3)) + [-1, 0, 2**31 - 1]:
            got, _ = ctx.run_host(_graph(c), E.make_opts(mode=E.THRESH_EXPLICIT, threshold=int(t)))
            assert np.array_equal(got, c["inMST"]), (name, t)


def test_heuristic_threshold_on_device_matches_reference(ctx, golden):
    for name, c in golden.items():
        if len(c["nlist"]) == 0:
            continue
        _, st = ctx.run_host(_graph(c))
        t, f = (int(x) for x in c["threshold"])
        assert (st["threshold"], st["filtered"]) == (t, f), name


def _families():
    return [
        ("grid_c1", lambda: E.gen_grid(1000, 1000, 1, 1_000_000)),
        ("rmat16", lambda: E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 2, 1 << 24)),
        ("rmat18_ef8", lambda: E.gen_rmat(18, 8, 0.57, 0.19, 0.19, 21, 1 << 20)),
        ("er", lambda: E.gen_er(200_000, 8, 5, 1 << 20)),
        ("er_dense", lambda: E.gen_er(50_000, 32, 6, 1 << 30)),
        ("rgg", lambda: E.gen_rgg2d(300_000, 3, 7, 1 << 20)),
        ("grid_ties", lambda: E.gen_grid(300, 700, 3, 4)),
    ]


@pytest.mark.parametrize("name,make", _families(), ids=[f[0] for f in _families()])
def test_generated_families_vs_oracle(ctx, name, make):
    g = make()
    t, f = E.heuristic_threshold(g)
    want, w, fe = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
    for kw in (dict(), dict(mode=E.THRESH_QUANTILE, quantile=0.1), dict(mode=E.THRESH_NONE),
               dict(degree_split=8)):
        got, st = ctx.run_host(g, E.make_opts(**kw))
        assert st["status"] == 0
        assert np.array_equal(got, want), (name, kw)
        assert st["forest_weight"] == w and st["forest_edges"] == fe


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name,make", _families()[:4], ids=[f[0] for f in _families()[:4]])
def test_vs_reference_rebuilt_for_sm100a(ctx, name, make):
    g = make()
    t, f = O.ref_threshold(g.nodes, g.eweight)
    ref_out, _ = O.ref_gpu_mst(g.nindex, g.nlist, g.eweight, f, t)
    got, _ = ctx.run_host(g)
    assert np.array_equal(got, ref_out), name


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")
def test_negative_weights_follow_reference_gpu(ctx):
    """With negative weights the reference GPU path orders weights as uint32
    and splits phases by a signed compare; the default schedule reproduces it."""
    rng = np.random.default_rng(7)
    for s in range(4):
        g = E.gen_er(3000, 10, 100 + s, 1000)
        g.eweight = (g.eweight - 500).astype(np.int32)  # mirrored, some negative
        t, f = O.ref_threshold(g.nodes, g.eweight)
        ref_out, _ = O.ref_gpu_mst(g.nindex, g.nlist, g.eweight, f, t)
        got, _ = ctx.run_host(g)
        assert np.array_equal(got, ref_out)
        ours, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
        assert np.array_equal(ours, ref_out)


def test_device_entry_point_with_torch_buffers(ctx):
    import torch
    g = E.gen_rmat(15, 16, 0.57, 0.19, 0.19, 9, 1 << 24)
    want, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, *E.heuristic_threshold(g))
    dev = torch.device("cuda:0")
    ni = torch.from_numpy(g.nindex).to(dev)
    nl = torch.from_numpy(g.nlist).to(dev)
    ew = torch.from_numpy(g.eweight).to(dev)
    out = torch.empty(g.edges, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        out.fill_(7)
        # torch's default stream is handle 0, which the library reads as the
        # context's own stream: wait for torch's work before the solve
        torch.cuda.synchronize()
        ctx.run_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(),
                       stream=s)
        torch.cuda.synchronize()
        ctx.sync()
        assert np.array_equal(out.cpu().numpy(), want)


def test_context_reuse_across_graphs(ctx, golden):
    names = list(golden)
    for name in names + names[::-1]:
        c = golden[name]
        got, _ = ctx.run_host(_graph(c))
        assert np.array_equal(got, c["inMST"]), name


def test_out_of_range_neighbour_is_reported_not_read(ctx):
    g = E.gen_grid(50, 50, 1, 100)
    nl = g.nlist.copy()
    nl[17] = g.nodes + 5
    with pytest.raises(E.EclError) as ei:
        ctx.run_host(E.Graph(g.nindex, nl, g.eweight))
    assert ei.value.status == -3
    ni = g.nindex.copy()
    ni[10] = g.edges + 100  # row beyond the edge array
    with pytest.raises(E.EclError) as ei:
        ctx.run_host(E.Graph(ni, g.nlist, g.eweight))
    assert ei.value.status == -3
    got, _ = ctx.run_host(g)  # the context stays usable
    want, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight)
    assert np.array_equal(got, want)


def test_too_large_for_context(ctx):
    small = E.Context(100, 100)
    g = E.gen_grid(20, 20, 1, 100)
    with pytest.raises(E.EclError) as ei:
        small.run_host(g)
    assert ei.value.status == -9
    small.close()


def test_stats_are_consistent(ctx):
    g = E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 2, 1 << 24)
    _, st = ctx.run_host(g, E.make_opts(flags=E.FLAG_STATS))
    assert st["filtered"] == 1 and st["rounds"][0] > 0 and st["rounds"][1] > 0
    # the light scan keeps exactly the one-direction entries with w <= threshold
    # (its worklist may add null padding after them, at most 63 slots per scan warp)
    row = np.repeat(np.arange(g.nodes), np.diff(g.nindex))
    light = int(np.count_nonzero((g.nlist > row) & (g.eweight <= st["threshold"])))
    assert st["scan_kept"][0] == light
    assert light <= st["wl_in"][0][0] <= light + 148 * 4 * 8 * 63
    assert 0 < st["scan_kept"][1] <= st["wl_in"][1][0]
    # rounds: the real entries never grow; round 0's slots also hold the scan's null padding
    for p in range(2):
        real, slots = st["wl_real"][p], st["wl_in"][p]
        assert real[0] == st["scan_kept"][p]
        for r in range(st["rounds"][p]):
            assert real[r] <= slots[r]
            if r + 1 <= st["rounds"][p] and r + 1 < len(real):
                assert real[r + 1] <= real[r]
    assert st["atomics"] > 0
    assert st["ms_total"] > 0
    assert st["forest_edges"] <= g.nodes - 1


@pytest.mark.slow
def test_rmat22_full_size_vs_oracle(ctx):
    """The single-graph benchmark input (RMAT scale 22, edge factor 16, seed 2)."""
    g = E.gen_rmat(22, 16, 0.57, 0.19, 0.19, 2, 1 << 24)
    big = E.Context(g.nodes, g.edges)
    t, f = E.heuristic_threshold(g)
    want, w, fe = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
    for kw in (dict(), dict(mode=E.THRESH_QUANTILE, quantile=0.05)):
        got, st = big.run_host(g, E.make_opts(**kw))
        assert np.array_equal(got, want), kw
        assert st["forest_weight"] == w
    big.close()


def _csr_from_edges(n, u, v, w):
    """Symmetric CSR (rows sorted by neighbour) from undirected edge arrays."""
    src = np.concatenate([u, v]).astype(np.int64)
    dst = np.concatenate([v, u]).astype(np.int64)
    wt = np.concatenate([w, w]).astype(np.int32)
    order = np.lexsort((dst, src))
    src, dst, wt = src[order], dst[order], wt[order]
    nindex = np.zeros(n + 1, np.int32)
    np.add.at(nindex, src + 1, 1)
    return E.Graph(np.cumsum(nindex).astype(np.int32), dst.astype(np.int32), wt)


def test_long_zero_degree_runs(ctx):
    """Tiles whose rows span more vertices than the staged nindex slice holds
    (runs of thousands of isolated vertices between dense clusters) take the
    global-search path; clusters of short rows between them take the staged one."""
    rng = np.random.default_rng(5)
    n = 300_000
    clusters = [np.arange(0, 3000), np.arange(40_000, 40_050), np.arange(150_000, 152_000),
                np.arange(299_000, 300_000)]
    us, vs = [], []
    for c in clusters:
        k = len(c) * 6
        us.append(rng.choice(c, k))
        vs.append(rng.choice(c, k))
    # a few long-range edges joining the clusters, and a hub
    us.append(np.array([5, 40_010, 150_500, 299_999] + [7] * 500))
    vs.append(np.array([40_020, 150_700, 299_500, 6] + list(rng.choice(n, 500))))
    u, v = np.concatenate(us), np.concatenate(vs)
    keep = u != v
    u, v = u[keep], v[keep]
    lo, hi = np.minimum(u, v), np.maximum(u, v)
    pairs = np.unique(lo.astype(np.int64) * n + hi)
    u, v = (pairs // n).astype(np.int64), (pairs % n).astype(np.int64)
    w = rng.integers(1, 1000, len(u)).astype(np.int32)  # many ties
    g = _csr_from_edges(n, u, v, w)
    for kw in (dict(degree_split=1), dict(degree_split=8), dict(degree_split=1 << 20),
               dict(mode=E.THRESH_NONE), dict(mode=E.THRESH_QUANTILE, quantile=0.3)):
        o = E.make_opts(**kw)
        got, st = ctx.run_host(g, o)
        t, f = st["threshold"], st["filtered"]
        want, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
        assert np.array_equal(got, want), kw


def test_unaligned_device_buffers(ctx):
    """CSR arrays and inMST starting 4 bytes past a 16-byte boundary: the scans
    stage them with plain copies instead of bulk copies."""
    import torch
    g = E.gen_rmat(14, 16, 0.57, 0.19, 0.19, 4, 1 << 20)
    want, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, *E.heuristic_threshold(g))
    dev = torch.device("cuda:0")

    def shifted(a):
        buf = torch.zeros(len(a) + 1, dtype=torch.int32, device=dev)
        buf[1:] = torch.from_numpy(a).to(dev)
        return buf, buf[1:].data_ptr()

    (bi, ni), (bl, nl), (bw, ew) = shifted(g.nindex), shifted(g.nlist), shifted(g.eweight)
    out = torch.zeros(g.edges + 1, dtype=torch.uint8, device=dev)
    for split in (1, 8, 1 << 20):
        out.fill_(7)
        ctx.run_device(g.nodes, g.edges, ni, nl, ew, out[1:].data_ptr(), opts=E.make_opts(degree_split=split))
        ctx.sync()
        got = out.cpu().numpy()
        assert got[0] == 7 and np.array_equal(got[1:], want), split


def test_cli_variants_and_table_pipeline(tmp_path):
    """The drop-in CLI prints the reference binary's blocks (input line + one
    runtime per run) for each deoptimized variant it reproduces; the table port
    reads them; every variant reports the same forest."""
    import os
    import subprocess
    import compare_tables as T
    exe = os.path.join(os.path.dirname(E.LIB_PATH), "ecl_mst")
    g = E.gen_rmat(14, 16, 0.57, 0.19, 0.19, 5, 1 << 20)
    path = str(tmp_path / "rmat14.egr")
    E.write_graph(g, path)
    outs, forests = {}, set()
    # the reference's variant chain (generate_deoptimize_tables.py:6-14)
    for v in ("base", "NAG", "NAG_NW", "NAG_NW_NF", "NAG_NW_NF_NIPC", "NAG_NW_NF_NIPC_NOD",
              "NAG_NW_NF_NIPC_NOD_NT", "NAG_NW_NF_NIPC_NOD_NT_NDD", "NAG_NW_NF_NIPC_NOD_NT_NDD_NEB"):
        r = subprocess.run([exe, path, "3", v], capture_output=True, text=True, timeout=120)
        assert r.returncode == 0, r.stderr
        assert ("NOD" in v) == ("NOD is not reproduced" in r.stderr)
        outs[f"ecl_mst_{v}_out.csv"] = r.stdout
        forests.add(r.stdout.strip().splitlines()[-1])
    assert len(forests) == 1
    inputs, names, rt, tp = T.tables(outs, runs=3)
    assert len(inputs) == 1 and all(x is not None and x > 0 for x in tp[0])
    r = subprocess.run([exe, path, "3", "NAG_XYZ"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0


def test_repeated_solve_is_captured_and_replayed(ctx):
    """A solve repeated on the same buffers and options is captured as a CUDA
    graph on the first repeat and replayed after that; the replay reads the
    buffers afresh, so changed weights give the new forest."""
    import torch
    g = E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 12, 1 << 20)
    dev = torch.device("cuda:0")
    ni = torch.from_numpy(g.nindex).to(dev)
    nl = torch.from_numpy(g.nlist).to(dev)
    ew = torch.from_numpy(g.eweight).to(dev)
    out = torch.empty(g.edges, dtype=torch.uint8, device=dev)
    s = torch.cuda.current_stream().cuda_stream
    E.learned_load_default()
    for kw in (dict(), dict(mode=E.THRESH_LEARNED)):
        o = E.make_opts(**kw)
        for step in range(4):
            w = g.eweight if step < 3 else (g.eweight ^ 0x5A5A).astype(np.int32)
            ew.copy_(torch.from_numpy(w))
            out.fill_(7)
            torch.cuda.synchronize()  # torch's stream (handle 0) is not the one the solve runs on
            st = ctx.run_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(),
                                opts=o, stream=s, stats=True)
            want, _, _ = O.oracle_mst(g.nindex, g.nlist, w, st["threshold"], st["filtered"])
            assert np.array_equal(out.cpu().numpy(), want), (kw, step)
            assert st["ms_total"] > 0 and st["status"] == 0


def _forward_only(n, k, seed):
    """Every undirected edge stored once, forward (nlist[j] > v): v -> v+1 .. v+k.
    All m entries are one-direction entries, twice what a symmetric input has."""
    v = np.repeat(np.arange(n - k, dtype=np.int64), k)
    nb = v + np.tile(np.arange(1, k + 1), n - k)
    nindex = np.zeros(n + 1, np.int32)
    nindex[1:] = np.cumsum(np.bincount(v, minlength=n))
    w = np.random.default_rng(seed).integers(1, 1 << 20, len(nb)).astype(np.int32)
    return E.Graph(nindex, nb.astype(np.int32), w)


@pytest.mark.parametrize("k", [3, 6])
def test_one_direction_input_grows_the_worklists(k):
    """Contexts size their worklists for symmetric input (edges/2 one-direction
    entries plus slack). An input with more overflows them; the library grows
    them and repeats the solve on each synchronising path: run_host, a device
    solve with stats, and a device solve checked by ctx_sync."""
    import torch
    g = _forward_only(1 << 20, k, 5 + k)
    t, f = E.heuristic_threshold(g)
    want, w, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
    with E.Context(g.nodes, g.edges) as c:
        got, st = c.run_host(g)
        assert st["status"] == 0 and np.array_equal(got, want) and st["forest_weight"] == w
    dev = torch.device("cuda:0")
    ni, nl, ew = (torch.from_numpy(a).to(dev) for a in (g.nindex, g.nlist, g.eweight))
    for stats in (True, False):
        with E.Context(g.nodes, g.edges) as c:
            out = torch.full((g.edges,), 7, dtype=torch.uint8, device=dev)
            torch.cuda.synchronize()
            c.run_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(),
                         stream=torch.cuda.current_stream().cuda_stream, stats=stats)
            c.sync()
            assert np.array_equal(out.cpu().numpy(), want), stats


def test_pipelined_host_solves_match_the_oracle():
    """run_host_async overlaps each graph's copy in with the previous solve
    and copy back; after wait() every output is the oracle's, including an
    input whose one-direction entries overflow the half-size worklists
    (solved again inside the wait)."""
    import torch
    graphs = [E.gen_rmat(16, 16, 0.57, 0.19, 0.19, 21, 1 << 24), E.gen_grid(300, 300, 22, 1000),
              _forward_only(1 << 20, 3, 23), E.gen_er(50_000, 10, 24, 1 << 20), E.gen_rmat(15, 8, 0.57, 0.19, 0.19, 25, 99)]
    wants = []
    for g in graphs:
        t, f = E.heuristic_threshold(g)
        wants.append(O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)[0])
    with E.Context(max(g.nodes for g in graphs), max(g.edges for g in graphs)) as c:
        for rep in range(2):
            outs = []
            for g in graphs:
                pinned = [torch.from_numpy(a).pin_memory().numpy() for a in (g.nindex, g.nlist, g.eweight)]
                hg = E.Graph(*pinned)
                outs.append(c.run_host_async(hg, E.make_opts(mode=E.THRESH_LEARNED if rep else E.THRESH_HEURISTIC),
                                             out=torch.full((g.edges,), 7, dtype=torch.uint8).pin_memory().numpy()))
            c.wait()
            for i, (got, want) in enumerate(zip(outs, wants)):
                assert np.array_equal(got, want), (rep, i)
