"""Host logic of the batched mode across GPUs (shard.py): the partition, and
the gather over a world-size-2 gloo process group on the CPU. Each rank
solves its shard with the CPU oracle here (no GPU): what is tested is that
every graph is solved exactly once and the gathered results equal a
single-process run."""
import os
import socket

import numpy as np
import pytest

import shard as S


def test_partition_covers_every_graph_once_and_balances():
    rng = np.random.default_rng(1)
    costs = (10 ** rng.uniform(3, 6.5, 300)).astype(np.int64)
    for world in (1, 2, 3, 8):
        shards = S.partition_by_cost(costs, world)
        ids = sorted(i for s in shards for i in s)
        assert ids == list(range(len(costs)))
        loads = [int(costs[s].sum()) if s else 0 for s in shards]
        # LPT bound: no rank above the mean by more than the largest graph
        assert max(loads) <= sum(loads) / world + costs.max()
    assert S.partition_by_cost(costs, 4) == S.partition_by_cost(costs, 4)
    assert S.partition_by_cost([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        S.partition_by_cost(costs, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    import ecl_mst as E
    import oracle_lib as O
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    graphs = [E.gen_batch_graph(i, nmin=200, nmax=3000)[0] for i in range(12)]
    shards = S.partition_by_cost([g.edges for g in graphs], world)
    local = {}
    for gid in shards[rank]:
        g = graphs[gid]
        _, w, fe = O.oracle_mst(g.nindex, g.nlist, g.eweight)
        local[gid] = (int(w), int(fe), rank)
    merged = S.gather_results(local, dist)
    np.save(os.path.join(out_dir, f"rank{rank}.npy"),
            np.array(sorted((k, v[0], v[1], v[2]) for k, v in merged.items()), dtype=np.int64))
    dist.destroy_process_group()


def test_gather_over_gloo_world_2(tmp_path):
    import torch.multiprocessing as mp
    import ecl_mst as E
    import oracle_lib as O
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r0, r1 = np.load(tmp_path / "rank0.npy"), np.load(tmp_path / "rank1.npy")
    assert np.array_equal(r0, r1)  # every rank holds the whole result
    assert sorted(r0[:, 0].tolist()) == list(range(12))
    assert set(r0[:, 3].tolist()) == {0, 1}  # both ranks did work
    for gid, w, fe, _ in r0:
        g, _ = E.gen_batch_graph(int(gid), nmin=200, nmax=3000)
        _, w1, fe1 = O.oracle_mst(g.nindex, g.nlist, g.eweight)
        assert (w, fe) == (int(w1), int(fe1))


def test_batch_view_of_a_shard_addresses_the_parent_layout():
    """A rank's shard as a view of the packed batch: the per-graph tables are
    the parent's rows in shard order, the entries and the output offsets stay
    the parent's, and the ecl_batch struct carries the view's tables."""
    import ecl_mst as E
    graphs = [E.gen_batch_graph(i, nmin=200, nmax=3000)[0] for i in range(10)]
    b = E.Batch(graphs)
    for world in (2, 3):
        for rank, mine in enumerate(S.partition_by_cost([g.edges for g in graphs], world)):
            v = b.select(mine)
            assert v.num_graphs == len(mine) and v.total_edges == b.total_edges
            for k, gid in enumerate(mine):
                assert (v.nodes[k], v.edges[k]) == (graphs[gid].nodes, graphs[gid].edges)
                assert (v.nindex_off[k], v.edge_off[k]) == (b.nindex_off[gid], b.edge_off[gid])
                a = int(b.edge_off[gid])
                assert np.array_equal(b.nlist[a:a + graphs[gid].edges], graphs[gid].nlist)
            out = np.arange(b.total_edges, dtype=np.int64)
            assert all(np.array_equal(v.slice(out, k), b.slice(out, gid)) for k, gid in enumerate(mine))
            st = v.struct(1, 2, 3)
            assert st.num_graphs == len(mine) and (st.nindex, st.nlist, st.eweight) == (1, 2, 3)
            assert st.edge_off == v.edge_off.ctypes.data
