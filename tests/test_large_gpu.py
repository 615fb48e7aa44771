"""Large single graphs (about 8 GB of CSR): RMAT scale 25 (33,554,432
vertices, edge factor 16, seed 3) and Erdos-Renyi with 16,777,216 vertices at
average degree 32 (seed 3), weights uniform in [1, 2^30]. The CUDA path under
the learned and the reference-heuristic schedules must give the inMST of the
reference's own gpuMST (ECL-MST/ECL_MST.cu:265-362) rebuilt for sm_100a, bit
for bit, and the same uint64 forest weight.

The inputs are drawn on the device by the library's generators (entry for
entry the host generators' graphs, tests/test_preprocess_gpu.py), which takes
well under a second; the reference gets a host copy."""
import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GRAPHS = {
    "rmat25": lambda: E.gen_rmat_device(25, 16, 0.57, 0.19, 0.19, 3, 1 << 30),
    "er16m": lambda: E.gen_er_device(1 << 24, 32, 3, 1 << 30),
}


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built")
@pytest.mark.parametrize("name", list(GRAPHS))
def test_large_graph_vs_reference_gpu(name):
    import torch
    dg = GRAPHS[name]()
    try:
        g = dg.to_host()
        t, f = O.ref_threshold(g.nodes, g.eweight)
        ref_out, _ = O.ref_gpu_mst(g.nindex, g.nlist, g.eweight, f, t)
        ref_w = int(g.eweight[ref_out.astype(bool)].astype(np.int64).sum()) % 2**64
        E.learned_load_default()
        out = torch.empty(g.edges, dtype=torch.uint8, device="cuda:0")
        with E.Context(g.nodes, g.edges) as ctx:
            for kw in (dict(), dict(mode=E.THRESH_LEARNED)):
                st = ctx.run_device(g.nodes, g.edges, dg.d_nindex, dg.d_nlist, dg.d_eweight, out.data_ptr(),
                                    opts=E.make_opts(**kw), stats=True)
                assert st["status"] == 0
                got = out.cpu().numpy()
                assert np.array_equal(got, ref_out), (name, kw)
                assert int(g.eweight[got.astype(bool)].astype(np.int64).sum()) % 2**64 == ref_w
        del out
    finally:
        dg.close()
