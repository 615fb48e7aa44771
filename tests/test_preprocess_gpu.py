"""GPU-side preprocessing: the device generators give the host generators'
graphs entry for entry; the pair-list CSR builder deduplicates, symmetrises
and drops self-loops like a numpy restatement, keeps the smallest uint32
weight of duplicate pairs, and synthesises the reference's weights for
weightless inputs (ECL_MST.cu:410-419); device-built graphs and batches solve
to the oracle's forest."""
import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0")


def _same(a, b):
    assert a.nodes == b.nodes and a.edges == b.edges
    assert np.array_equal(a.nindex, b.nindex)
    assert np.array_equal(a.nlist, b.nlist)
    assert np.array_equal(a.eweight, b.eweight)


@pytest.mark.parametrize("rows,cols", [(1, 1), (1, 7), (9, 1), (2, 2), (31, 17), (300, 301)])
def test_grid_device_equals_host(rows, cols):
    with E.gen_grid_device(rows, cols, 5, 1000) as d:
        _same(d.to_host(), E.gen_grid(rows, cols, 5, 1000))


@pytest.mark.parametrize("nodes,deg", [(1, 4.0), (2, 1.0), (1000, 0.0), (5000, 8.0), (200000, 8.0)])
def test_er_device_equals_host(nodes, deg):
    with E.gen_er_device(nodes, deg, 17, 1 << 20) as d:
        _same(d.to_host(), E.gen_er(nodes, deg, 17, 1 << 20))


@pytest.mark.parametrize("scale,ef", [(1, 4), (5, 16), (12, 8), (16, 16)])
def test_rmat_device_equals_host(scale, ef):
    with E.gen_rmat_device(scale, ef, 0.57, 0.19, 0.19, 2, 1 << 24) as d:
        _same(d.to_host(), E.gen_rmat(scale, ef, 0.57, 0.19, 0.19, 2, 1 << 24))


@pytest.mark.parametrize("nodes,deg", [(1, 3.0), (7, 3.0), (5000, 3.0), (100000, 3.0), (20000, 20.0)])
def test_rgg2d_device_equals_host(nodes, deg):
    with E.gen_rgg2d_device(nodes, deg, 9, 1 << 20) as d:
        _same(d.to_host(), E.gen_rgg2d(nodes, deg, 9, 1 << 20))


@pytest.mark.parametrize("index", list(range(0, 40, 3)))
def test_batch_graph_device_equals_host(index):
    d, fam_d = E.gen_batch_graph_device(index, nmax=200_000)
    h, fam_h = E.gen_batch_graph(index, nmax=200_000)
    assert fam_d == fam_h
    _same(d.to_host(), h)
    d.close()


def _csr_ref(n, u, v, w):
    """numpy restatement: both directions of every non-loop pair, sorted by
    (row, neighbour), one entry per distinct pair, weight = the smallest of
    its duplicates as uint32."""
    u = u.astype(np.int64)
    v = v.astype(np.int64)
    keep = u != v
    a = np.concatenate([u[keep], v[keep]])
    b = np.concatenate([v[keep], u[keep]])
    ww = np.concatenate([w[keep], w[keep]]).view(np.uint32).astype(np.int64)
    key = a * n + b
    order = np.lexsort((ww, key))
    key, ww = key[order], ww[order]
    head = np.ones(len(key), bool)
    head[1:] = key[1:] != key[:-1]
    rows, cols = key[head] // n, key[head] % n
    nindex = np.zeros(n + 1, np.int64)
    np.add.at(nindex, rows + 1, 1)
    return (np.cumsum(nindex).astype(np.int32), cols.astype(np.int32),
            ww[head].astype(np.uint32).view(np.int32))


def test_pairs_given_weights_dedup_symmetrise_and_keep_the_uint32_minimum():
    rng = np.random.default_rng(5)
    n, p = 3000, 60000
    u = rng.integers(0, 400, p).astype(np.int32)  # a narrow range forces many duplicates
    v = rng.integers(0, n, p).astype(np.int32)
    v[::7] = u[::7]  # self-loops
    v[1::11], u[1::11] = u[1::11].copy(), v[1::11].copy()  # both orientations of one pair
    w = rng.integers(-(2 ** 31), 2 ** 31, p).astype(np.int32)
    du, dv, dw = _dev(u), _dev(v), _dev(w)
    with E.csr_from_pairs_device(n, p, du.data_ptr(), dv.data_ptr(), dw.data_ptr(), E.WEIGHTS_GIVEN) as d:
        g = d.to_host()
    ni, nl, ew = _csr_ref(n, u, v, w)
    assert np.array_equal(g.nindex, ni) and np.array_equal(g.nlist, nl) and np.array_equal(g.eweight, ew)
    # symmetric weights: entry (a, b) and (b, a) agree
    rows = np.repeat(np.arange(n), np.diff(g.nindex))
    fwd = dict(zip(zip(rows.tolist(), g.nlist.tolist()), g.eweight.tolist()))
    assert all(fwd[(b, a)] == x for (a, b), x in fwd.items())


def test_pairs_synth_rule_is_the_reference_weight_synthesis():
    rng = np.random.default_rng(6)
    n, p = 70000, 300000  # i * k wraps int32 for ids this large
    u = rng.integers(0, n, p).astype(np.int32)
    v = rng.integers(0, n, p).astype(np.int32)
    du, dv = _dev(u), _dev(v)
    with E.csr_from_pairs_device(n, p, du.data_ptr(), dv.data_ptr(), None, E.WEIGHTS_SYNTH) as d:
        g = d.to_host()
    ni, nl, _ = _csr_ref(n, u, v, np.zeros(p, np.int32))
    assert np.array_equal(g.nindex, ni) and np.array_equal(g.nlist, nl)
    want = E.synthesize_weights(E.Graph(g.nindex, g.nlist, None))
    assert np.array_equal(g.eweight, want.eweight)


@pytest.mark.parametrize("case", ["no_pairs", "only_loops", "one_pair", "one_vertex"])
def test_pairs_edge_cases(case):
    n, u, v = {"no_pairs": (10, [], []), "only_loops": (10, [3, 3, 9], [3, 3, 9]),
               "one_pair": (5, [4], [0]), "one_vertex": (1, [0], [0])}[case]
    u, v = np.array(u, np.int32), np.array(v, np.int32)
    w = np.full(len(u), 5, np.int32)
    du, dv, dw = _dev(u), _dev(v), _dev(w)
    with E.csr_from_pairs_device(n, len(u), du.data_ptr() if len(u) else None, dv.data_ptr() if len(u) else None,
                                 dw.data_ptr() if len(u) else None, E.WEIGHTS_GIVEN) as d:
        g = d.to_host()
    ni, nl, ew = _csr_ref(n, u, v, w)
    assert np.array_equal(g.nindex, ni) and np.array_equal(g.nlist, nl) and np.array_equal(g.eweight, ew)


@pytest.mark.parametrize("bad", [10, -1])
def test_pairs_out_of_range_id_is_a_format_error(bad):
    u = np.array([0, 1, bad, 2], np.int32)
    v = np.array([1, 2, 3, 0], np.int32)
    du, dv = _dev(u), _dev(v)
    with pytest.raises(E.EclError) as ei:
        E.csr_from_pairs_device(10, 4, du.data_ptr(), dv.data_ptr(), None, E.WEIGHTS_HASH, 1, 100)
    assert ei.value.status == -3


def test_device_generated_graph_solves_to_the_oracle_forest():
    import torch
    with E.gen_rmat_device(15, 16, 0.57, 0.19, 0.19, 2, 1 << 24) as d:
        h = d.to_host()
        out = torch.zeros(d.edges, dtype=torch.uint8, device="cuda:0")
        torch.cuda.synchronize()
        with E.Context(d.nodes, d.edges) as ctx:
            ctx.run_device(d.nodes, d.edges, d.d_nindex, d.d_nlist, d.d_eweight, out.data_ptr(),
                           stream=torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
        got = out.cpu().numpy()
    t, f = E.heuristic_threshold(h)
    want, w, fe = O.oracle_mst(h.nindex, h.nlist, h.eweight, t, f)
    assert np.array_equal(got, want)


def test_device_batch_packs_the_host_batch_and_solves_identically():
    import torch
    count, nmax = 40, 100_000
    db = E.DeviceBatch(count, nmax=nmax)
    graphs = [E.gen_batch_graph(i, nmax=nmax)[0] for i in range(count)]
    hb = E.Batch(graphs)
    assert np.array_equal(db.nodes, hb.nodes) and np.array_equal(db.edges, hb.edges)
    assert np.array_equal(db.nindex_off, hb.nindex_off) and np.array_equal(db.edge_off, hb.edge_off)
    assert db.total_edges == hb.total_edges and db.total_nindex == hb.total_nindex
    for i in (0, 1, 17, count - 1):
        _same(db.graph(i), graphs[i])
    out = torch.zeros(db.total_edges, dtype=torch.uint8, device="cuda:0")
    bc = E.BatchContext(count, int(db.nodes.max()), int(db.edges.max()))
    st = bc.run(db, db.d_nindex, db.d_nlist, db.d_eweight, out.data_ptr())
    assert st["status"] == 0
    got = out.cpu().numpy()
    for i, g in enumerate(graphs):
        t, f = E.heuristic_threshold(g) if g.edges else (2 ** 31 - 1, 0)
        want = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)[0]
        assert np.array_equal(db.slice(got, i), want[: g.edges]), i
    bc.close()
    db.close()
