"""The table pipeline's median / throughput computation over ecl_mst output
(compare_tables.py, restating generate_compare_tables.py:39-63). CPU only."""
import os
import statistics

import numpy as np

import compare_tables as T
import ecl_mst as E


def _block(path, vals, trailer=True):
    s = f"input: {path}\n" + "".join(f"{v:12.9f}\n" for v in vals)
    return s + ("forest: 3 edges, weight 7\n" if trailer else "")


def test_parse_and_medians_match_the_reference_rule():
    a = [0.5, 0.1, 0.3, 0.2, 0.9, 0.4, 0.7, 0.6, 0.8]
    b = [1.0] * 9
    text = "Deoptimized runs\n" + _block("inputs/rmat16.sym.egr", a) + _block("inputs/internet.egr", b)
    blocks = T.parse_runs(text)
    assert [p for p, _ in blocks] == ["inputs/rmat16.sym.egr", "inputs/internet.egr"]
    sizes = {"rmat16.sym": 967866, "internet": 387240}
    inputs, names, rt, tp = T.tables({"ecl_mst_out.csv": text}, sizes)
    assert names == ["ecl_mst_out.csv"]
    assert rt[0][0] == statistics.median(a) and rt[1][0] == 1.0
    assert abs(tp[0][0] - 967866 / statistics.median(a) / 1e6) < 1e-9
    assert abs(tp[1][0] - 0.38724) < 1e-12


def test_two_outputs_and_missing_inputs(tmp_path):
    base = _block("g1.egr", [2.0] * 9) + _block("g2.egr", [4.0] * 9)
    nag = _block("g1.egr", [3.0] * 9)
    inputs, names, rt, tp = T.tables({"ecl_mst_out.csv": base, "ecl_mst_NAG_out.csv": nag},
                                     {"g1": 2_000_000, "g2": 4_000_000})
    assert rt == [[2.0, 3.0], [4.0, None]]
    assert tp[0] == [1.0, 2.0 / 3.0] and tp[1][1] is None
    out = tmp_path / "t.csv"
    T.write_csv(str(out), inputs, names, rt)
    lines = out.read_text().splitlines()
    assert lines[0] == ",ecl_mst, ecl_mst_NAG, "
    assert lines[1] == "g1,2.0,3.0" and lines[2] == "g2,4.0,"


def test_sizes_from_the_graph_header(tmp_path):
    g = E.gen_grid(10, 12, 1, 100)
    path = str(tmp_path / "grid.egr")
    E.write_graph(g, path)
    inputs, _, rt, tp = T.tables({"o": _block(path, [0.001] * 9)})
    assert abs(tp[0][0] - g.edges / 0.001 / 1e6) < 1e-9
    assert os.path.basename(inputs[0]) == "grid.egr"


def test_only_the_first_runs_count():
    vals = [1.0] * 9 + [100.0] * 5
    _, _, rt, _ = T.tables({"o": _block("x.egr", vals)}, {"x": 10}, runs=9)
    assert rt[0][0] == 1.0
    _, _, rt, _ = T.tables({"o": _block("x.egr", vals)}, {"x": 10}, runs=None)
    assert rt[0][0] == float(np.median(vals))
