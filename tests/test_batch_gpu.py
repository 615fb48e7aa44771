"""Batched mode: many graphs of uneven sizes in one call, each bit-identical
to solving it alone (oracle), through the persistent one-CTA-per-graph launch
and the grid-wide engine (captured as a CUDA graph) for graphs beyond the
per-CTA cutoff."""
import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O

pytestmark = pytest.mark.gpu


def _mixed_graphs(seed0, count):
    rng = np.random.default_rng(seed0)
    gs = []
    for i in range(count):
        fam = i % 4
        n = int(np.exp(rng.uniform(np.log(50), np.log(60000))))
        s = seed0 + i
        if fam == 0:
            r = max(2, int(np.sqrt(n)))
            gs.append(E.gen_grid(r, max(1, n // r), s, 1 << 20))
        elif fam == 1:
            gs.append(E.gen_er(n, 8, s, 1 << 20))
        elif fam == 2:
            gs.append(E.gen_rmat(max(6, int(np.log2(n))), 8, 0.57, 0.19, 0.19, s, 1 << 20))
        else:
            gs.append(E.gen_rgg2d(n, 3, s, 1 << 20))
    gs.append(E.Graph(np.array([0, 0], np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)))  # 1 vertex
    return gs


def _run(graphs, small_cap, opts_list):
    import torch
    b = E.Batch(graphs)
    dev = torch.device("cuda:0")
    ni = torch.from_numpy(b.nindex).to(dev)
    nl = torch.from_numpy(b.nlist).to(dev)
    ew = torch.from_numpy(b.eweight).to(dev)
    out = torch.zeros(b.total_edges, dtype=torch.uint8, device=dev)
    bc = E.BatchContext(len(graphs), max(g.nodes for g in graphs), max(g.edges for g in graphs), small_cap)
    wants = []
    for g in graphs:
        t, f = E.heuristic_threshold(g) if g.edges else (2**31 - 1, 0)
        wants.append(O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)[0])
    results = []
    for o in opts_list:
        for rep in range(2):  # second run replays the captured large-graph sequence
            out.fill_(3)
            st = bc.run(b, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(), opts=o)
            got = out.cpu().numpy()
            for gi, g in enumerate(graphs):
                assert np.array_equal(b.slice(got, gi), wants[gi]), (gi, g.nodes, g.edges, rep)
            results.append(st)
    bc.close()
    return results


def test_batch_all_small():
    sts = _run(_mixed_graphs(1000, 40), 1 << 19, [None])
    assert sts[0]["graphs_large"] == 0 and sts[0]["status"] == 0


def test_batch_mixed_small_and_large():
    opts = [None, E.make_opts(mode=E.THRESH_QUANTILE, quantile=0.05, degree_split=16, small_tail=1024)]
    sts = _run(_mixed_graphs(2000, 40), 1 << 12, opts)
    assert all(s["graphs_large"] > 0 and s["graphs_small"] > 0 for s in sts)
    assert sts[1]["graph_replay"] == 1


@pytest.mark.parametrize("streams,cps", [(1, 0), (3, 0), (8, 2), (0, 0)])
def test_batch_large_graphs_on_concurrent_streams(streams, cps):
    """The graphs beyond the per-CTA cutoff spread over 1, 3 or 8 concurrent
    streams (each with its own engine; largest first to the least-loaded
    stream) or the default; every graph keeps the oracle's forest, directly
    and from the replayed capture."""
    opts = [E.make_opts(batch_large_streams=streams, ctas_per_sm=cps),
            E.make_opts(mode=E.THRESH_QUANTILE, quantile=0.1, batch_large_streams=streams, ctas_per_sm=cps)]
    sts = _run(_mixed_graphs(5000, 40), 1 << 11, opts)
    assert all(s["graphs_large"] >= 8 and s["status"] == 0 for s in sts)
    assert sts[1]["graph_replay"] == 1 and sts[3]["graph_replay"] == 1


def test_batch_autotune_keeps_the_answer():
    import torch
    graphs = _mixed_graphs(3000, 16)
    b = E.Batch(graphs)
    dev = torch.device("cuda:0")
    ni = torch.from_numpy(b.nindex).to(dev)
    nl = torch.from_numpy(b.nlist).to(dev)
    ew = torch.from_numpy(b.eweight).to(dev)
    out = torch.zeros(b.total_edges, dtype=torch.uint8, device=dev)
    bc = E.BatchContext(len(graphs), max(g.nodes for g in graphs), max(g.edges for g in graphs), 1 << 13)
    best, ms = bc.autotune(b, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr())
    assert ms > 0 and best.batch_small_edges > 0
    bc.run(b, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(), opts=best)
    got = out.cpu().numpy()
    for gi, g in enumerate(graphs):
        t, f = E.heuristic_threshold(g) if g.edges else (2**31 - 1, 0)
        assert np.array_equal(b.slice(got, gi), O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)[0])
    bc.close()


def test_batch_learned_schedule_on_large_graphs():
    """Large graphs of a batch (beyond the per-CTA cutoff, at least 2^20 CSR
    entries) take the learned schedule, feature pass on a side stream inside
    the captured launch sequence; every graph keeps the oracle's forest."""
    if not E.learned_load_default():
        pytest.skip("no trained weights shipped")
    graphs = _mixed_graphs(4000, 12) + [
        E.gen_rmat(17, 16, 0.57, 0.19, 0.19, 4101, 1 << 20), E.gen_er(200_000, 12, 4102, 1 << 20),
        E.gen_grid(700, 700, 4103, 1 << 20), E.gen_rgg2d(400_000, 3, 4104, 1 << 20)]
    sts = _run(graphs, 1 << 16, [E.make_opts(mode=E.THRESH_LEARNED)])
    assert all(s["graphs_large"] >= 4 and s["status"] == 0 for s in sts)


def test_shard_views_of_a_device_batch_solve_like_the_whole_batch():
    """Each rank of a multi-GPU batch run solves a view of its shard of the
    device-drawn batch (DeviceBatch.select): the shard's graphs get the whole
    batch's answer at the same offsets, and no other entry is written."""
    import shard as S
    import torch
    db = E.DeviceBatch(48, nmin=200, nmax=200_000)
    out_all = torch.zeros(db.total_edges, dtype=torch.uint8, device="cuda:0")
    bc = E.BatchContext(db.num_graphs, int(db.nodes.max()), int(db.edges.max()), 1 << 14)
    bc.run(db, db.d_nindex, db.d_nlist, db.d_eweight, out_all.data_ptr())
    want = out_all.cpu().numpy()
    bc.close()
    for gi in (0, 7, 47):  # spot checks against the oracle
        g = db.graph(gi)
        t, f = E.heuristic_threshold(g) if g.edges else (2**31 - 1, 0)
        assert np.array_equal(db.slice(want, gi), O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)[0])
    for mine in S.partition_by_cost([int(x) for x in db.edges], 3):
        v = db.select(mine)
        out = torch.full((db.total_edges,), 3, dtype=torch.uint8, device="cuda:0")
        bcv = E.BatchContext(v.num_graphs, int(v.nodes.max()), int(v.edges.max()), 1 << 14)
        for rep in range(2):  # the second run replays the captured sequence
            bcv.run(v, None, None, None, out.data_ptr())
            got = out.cpu().numpy()
            for k, gi in enumerate(mine):
                assert np.array_equal(v.slice(got, k), db.slice(want, gi)), (gi, rep)
            for gi in set(range(db.num_graphs)) - set(mine):  # other ranks' graphs: untouched
                assert (db.slice(got, gi) == 3).all(), (gi, rep)
        bcv.close()
    db.close()
