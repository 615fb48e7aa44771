"""The allocation-free entry point (ecl_mst_run_device_noalloc).

It exists for callers that cannot allocate device memory, for example code
running inside an allocator or memory-pool callback, or a process whose
device memory is owned by its host application. It keeps its scratch in a
static device array of the library. Its results must be bit-identical to the
ordinary device entry point on the same inputs, and a second call in a row
must not be disturbed by what the first one left in that array. This file is
collected last so a failure here does not hide the other tests' results.
"""
import numpy as np
import pytest

import ecl_mst as E

pytestmark = pytest.mark.gpu


def _to_dev(g, torch):
    dev = torch.device("cuda:0")
    return (torch.from_numpy(g.nindex).to(dev), torch.from_numpy(g.nlist).to(dev),
            torch.from_numpy(g.eweight).to(dev))


def test_noalloc_matches_device_entry_point_twice_in_a_row():
    import torch
    graphs = [E.gen_rmat(16, 8, 0.57, 0.19, 0.19, 31, 1 << 20),  # filtered, two phases
              E.gen_grid(300, 300, 32, 1000)]                    # unfiltered, one phase
    ctx = E.Context(max(g.nodes for g in graphs), max(g.edges for g in graphs))
    stream = torch.cuda.current_stream().cuda_stream
    for g in graphs:
        ni, nl, ew = _to_dev(g, torch)
        want_dev = torch.empty(g.edges, dtype=torch.uint8, device="cuda:0")
        ctx.run_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), want_dev.data_ptr(),
                       stream=stream)
        torch.cuda.synchronize()
        ctx.sync()
        want = want_dev.cpu().numpy()
        for _ in range(2):  # two calls in a row share the static scratch
            out = torch.full((g.edges,), 7, dtype=torch.uint8, device="cuda:0")
            E.run_device_noalloc(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr(),
                                 stream=stream)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.array_equal(got, want)
    ctx.close()


def test_noalloc_rejects_sizes_beyond_its_maximum():
    g = E.EclGraphC(1 << 19, 8, 1, 1, 1)  # never dereferenced: the size check comes first
    import ctypes
    st = E.load().ecl_mst_run_device_noalloc(ctypes.byref(g), 1, None, None)
    assert st == -9


def _csr_from_pairs(n, lo, hi, w):
    """Symmetric CSR (rows sorted by neighbour id) from distinct undirected
    pairs lo < hi with weights w, both directions carrying the pair's weight."""
    u = np.concatenate([lo, hi]).astype(np.int64)
    v = np.concatenate([hi, lo]).astype(np.int64)
    ww = np.concatenate([w, w]).astype(np.int32)
    order = np.lexsort((v, u))
    u, v, ww = u[order], v[order], ww[order]
    nindex = np.zeros(n + 1, np.int32)
    nindex[1:] = np.cumsum(np.bincount(u, minlength=n))
    return nindex, v.astype(np.int32), ww


def _max_size_graph():
    """Exactly the entry point's maximum: 262,144 vertices and 1,048,576
    directed CSR entries, a 512 x 512 grid (1,046,528 entries) plus 1,024
    distinct long-range edges, weights uniform in [1, 2^20] from a fixed seed."""
    rng = np.random.default_rng(123)
    side = 512
    n = side * side
    ids = np.arange(n).reshape(side, side)
    lo = np.concatenate([ids[:, :-1].ravel(), ids[:-1, :].ravel()])
    hi = np.concatenate([ids[:, 1:].ravel(), ids[1:, :].ravel()])
    have = set((lo.astype(np.int64) << 32 | hi).tolist())
    extra = []
    while len(extra) < 1024:
        a, b = sorted(rng.integers(0, n, 2).tolist())
        k = (a << 32) | b
        if a != b and k not in have:
            have.add(k)
            extra.append((a, b))
    lo = np.concatenate([lo, np.array([e[0] for e in extra])])
    hi = np.concatenate([hi, np.array([e[1] for e in extra])])
    w = rng.integers(1, (1 << 20) + 1, len(lo))
    return n, _csr_from_pairs(n, lo, hi, w)


def test_noalloc_at_its_maximum_size_matches_the_oracle():
    """At the stated maximum the scan's chunk slack is zero (the worklist
    holds exactly edges/2 entries); two calls in a row must both give the
    oracle's forest."""
    import torch
    import oracle_lib as O
    n, (nindex, nlist, eweight) = _max_size_graph()
    assert n == 1 << 18 and len(nlist) == 1 << 20
    t, f = O.oracle_heuristic(n, eweight)
    want, _, _ = O.oracle_mst(nindex, nlist, eweight, t, f)
    dev = torch.device("cuda:0")
    ni, nl, ew = (torch.from_numpy(a).to(dev) for a in (nindex, nlist, eweight))
    for _ in range(2):
        out = torch.full((len(nlist),), 7, dtype=torch.uint8, device=dev)
        E.run_device_noalloc(n, len(nlist), ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr())
        torch.cuda.synchronize()
        assert np.array_equal(out.cpu().numpy(), want)


def test_noalloc_explicit_threshold_and_learned_mode_match_run_device():
    import torch
    g = E.gen_rmat(15, 16, 0.57, 0.19, 0.19, 41, 1 << 20)
    ni, nl, ew = _to_dev(g, torch)
    with E.Context(g.nodes, g.edges) as ctx:
        for opts in (E.make_opts(mode=E.THRESH_EXPLICIT, threshold=1 << 14),
                     E.make_opts(mode=E.THRESH_LEARNED)):
            want = torch.empty(g.edges, dtype=torch.uint8, device="cuda:0")
            ctx.run_device(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), want.data_ptr(),
                           opts=opts, stats=True)
            got = torch.full((g.edges,), 7, dtype=torch.uint8, device="cuda:0")
            E.run_device_noalloc(g.nodes, g.edges, ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), got.data_ptr(),
                                 opts=opts)
            torch.cuda.synchronize()
            assert np.array_equal(got.cpu().numpy(), want.cpu().numpy())


def test_noalloc_reports_overflow_for_one_direction_input_beyond_its_worklist():
    """Every entry stored once, in the forward direction (nlist[j] > v):
    786,423 one-direction entries, more than the 524,288 the worklists hold."""
    import torch
    n = 1 << 18
    v = np.repeat(np.arange(n - 3, dtype=np.int64), 3)
    nb = v + np.tile(np.arange(1, 4), n - 3)
    nindex = np.zeros(n + 1, np.int32)
    nindex[1:] = np.cumsum(np.bincount(v, minlength=n))
    nlist = nb.astype(np.int32)
    eweight = (np.arange(len(nlist)) % 1000 + 1).astype(np.int32)
    dev = torch.device("cuda:0")
    ni, nl, ew = (torch.from_numpy(a).to(dev) for a in (nindex, nlist, eweight))
    out = torch.empty(len(nlist), dtype=torch.uint8, device=dev)
    with pytest.raises(E.EclError) as ei:
        E.run_device_noalloc(n, len(nlist), ni.data_ptr(), nl.data_ptr(), ew.data_ptr(), out.data_ptr())
    assert ei.value.status == -7
