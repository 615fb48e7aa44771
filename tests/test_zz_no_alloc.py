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
