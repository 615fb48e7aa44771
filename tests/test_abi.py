"""The C-ABI library: loads, exports every declared symbol, host-side logic
(graph I/O, validation, generators, heuristic, verify). No GPU needed."""
import ctypes
import os
import re

import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "ecl_mst.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = set(re.findall(r"\b(ecl_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = E.load()
    names = declared_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    assert E.load().ecl_version().startswith(b"ecl-mst-b200")


def test_status_strings():
    lib = E.load()
    for code in range(-10, 1):
        assert lib.ecl_status_string(code)


def test_graph_io_round_trip(tmp_path, golden):
    for name, c in list(golden.items())[:8]:
        g = E.Graph(c["nindex"], c["nlist"], c["eweight"])
        p = tmp_path / f"{name}.egr"
        E.write_graph(g, str(p))
        # byte layout: int32 nodes, edges, nindex, nlist, eweight
        raw = np.fromfile(p, np.int32)
        assert raw[0] == g.nodes and raw[1] == g.edges
        assert np.array_equal(raw[2:3 + g.nodes], g.nindex)
        h = E.read_graph(str(p))
        assert np.array_equal(h.nindex, g.nindex) and np.array_equal(h.nlist, g.nlist)
        if g.edges:
            assert np.array_equal(h.eweight, g.eweight)


def test_weightless_file_reads_null_weights(tmp_path):
    g = E.gen_grid(4, 5, 1, 10)
    p = tmp_path / "nw.egr"
    E.write_graph(E.Graph(g.nindex, g.nlist, None), str(p))
    h = E.read_graph(str(p))
    assert h.eweight is None and h.edges == g.edges


@pytest.mark.parametrize("cut", [0, 4, 9, 30])
def test_truncated_file_is_an_error(tmp_path, cut):
    g = E.gen_grid(4, 5, 1, 10)
    p = tmp_path / "t.egr"
    E.write_graph(g, str(p))
    data = p.read_bytes()
    q = tmp_path / "cut.egr"
    q.write_bytes(data[: 8 + cut * 4 // 2] if cut else data[:6])
    with pytest.raises(E.EclError) as ei:
        E.read_graph(str(q))
    assert ei.value.status == -3


def test_bad_counts_and_missing_file(tmp_path):
    q = tmp_path / "bad.egr"
    np.array([0, 5], np.int32).tofile(q)  # nodes < 1
    with pytest.raises(E.EclError):
        E.read_graph(str(q))
    np.array([3, -1], np.int32).tofile(q)  # edges < 0
    with pytest.raises(E.EclError):
        E.read_graph(str(q))
    with pytest.raises(E.EclError) as ei:
        E.read_graph(str(tmp_path / "nope.egr"))
    assert ei.value.status == -2


def test_validate_graph():
    g = E.gen_grid(3, 3, 1, 10)
    assert E.validate_graph(g) == 0
    bad = E.Graph(g.nindex, g.nlist.copy(), g.eweight)
    bad.nlist[3] = 9
    assert E.validate_graph(bad) == -3
    bad = E.Graph(g.nindex.copy(), g.nlist, g.eweight)
    bad.nindex[2], bad.nindex[3] = bad.nindex[3], bad.nindex[2]
    assert E.validate_graph(bad) == -3


def _check_symmetric(g):
    src = np.repeat(np.arange(g.nodes, dtype=np.int64), np.diff(g.nindex))
    assert (src != g.nlist).all(), "self-loop"
    k1 = (src << 32) | g.nlist
    k2 = (g.nlist.astype(np.int64) << 32) | src
    assert np.array_equal(np.sort(k1), np.sort(k2)), "not symmetric"
    assert np.array_equal(g.eweight[np.argsort(k1)], g.eweight[np.argsort(k2)]), "weights not mirrored"
    for v in range(min(g.nodes, 2000)):
        row = g.nlist[g.nindex[v]:g.nindex[v + 1]]
        assert (np.diff(row) > 0).all(), "row not sorted / duplicates"


def test_generators_shape_and_determinism():
    g = E.gen_grid(1000, 1000, 1, 1_000_000)
    assert (g.nodes, g.edges) == (1_000_000, 3_996_000)
    assert g.eweight.min() >= 1 and g.eweight.max() <= 1_000_000
    g2 = E.gen_grid(1000, 1000, 1, 1_000_000, threads=1)
    assert np.array_equal(g.eweight, g2.eweight)
    for gen in (lambda t: E.gen_rmat(14, 16, 0.57, 0.19, 0.19, 2, 1 << 24, t),
                lambda t: E.gen_er(20000, 8, 5, 1 << 20, t),
                lambda t: E.gen_rgg2d(20000, 3, 7, 1 << 20, t)):
        a, b = gen(0), gen(1)
        assert np.array_equal(a.nindex, b.nindex) and np.array_equal(a.nlist, b.nlist)
        assert np.array_equal(a.eweight, b.eweight)
        _check_symmetric(a)
        assert E.validate_graph(a) == 0


def test_rgg_average_degree_close():
    g = E.gen_rgg2d(200000, 3.0, 9, 1 << 20)
    assert 2.6 < g.edges / g.nodes < 3.1


def test_heuristic_matches_oracle(golden):
    for name, c in golden.items():
        if len(c["nlist"]) == 0:
            continue
        g = E.Graph(c["nindex"], c["nlist"], c["eweight"])
        assert E.heuristic_threshold(g) == tuple(int(x) for x in c["threshold"]), name


def test_verify_matches_oracle(golden):
    c = golden["grid_random"]
    g = E.Graph(c["nindex"], c["nlist"], c["eweight"])
    ok, counts, wa, wb = E.verify(g, c["inMST"], c["inMST"])
    assert ok and wa == wb
    bad = c["inMST"].copy()
    bad[np.flatnonzero(bad == 0)[0]] = 1
    ok, counts, wa, wb = E.verify(g, c["inMST"], bad)
    assert not ok and counts[3] == 1
    assert (ok, counts) == O.oracle_verify(c["eweight"], c["inMST"], bad)


def test_synthesize_weights_matches_oracle():
    g = E.gen_er(3000, 6, 3, 10)
    w = O.oracle_synth(g.nindex, g.nlist)
    E.synthesize_weights(g)
    assert np.array_equal(g.eweight, w)


def test_solve_rejects_bad_arguments_without_touching_a_device():
    g = E.gen_grid(3, 3, 1, 10)
    bad = E.Graph(np.array([0], np.int32), np.zeros(0, np.int32), None)  # nodes = 0
    with pytest.raises(E.EclError) as ei:
        E.mst(bad)
    assert ei.value.status == -1
    lib = E.load()
    o = E.make_opts(mode=99)
    gs = g.struct()
    out = np.zeros(g.edges, np.uint8)
    st = lib.ecl_mst_run(ctypes.byref(gs), out.ctypes.data_as(ctypes.c_void_p), ctypes.byref(o), None)
    assert st in (-1, -6)  # invalid option, or no device on this machine


def test_context_without_device_reports_no_device():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(E.EclError) as ei:
        E.Context(10, 10)
    assert ei.value.status == -6
