"""Generate tests/golden/converters.npz: inputs and outputs of the reference's
input converters, the checker of the library's text exporters.

The converters PBBS_CPU/inputs/ecl2pbbs_genweights.cpp and
cuGraph_GPU/inputs/ecl2mtx_genweights_cugraph.cpp are compiled unmodified
from the reference tree by `make -C oracle converters` into oracle/_ref/.
Each case is a small ECLgraph built here from a fixed seed, written as .egr,
converted by both reference binaries; the fixture stores the CSR arrays and
the two output files' bytes. Run from the repository root:

    make -C oracle converters && python tests/golden/make_converter_golden.py

Cases: weights from the generator; extreme weights (INT32_MIN, INT32_MAX, 0,
2^24 + 1, which float rounds, and random 32-bit values); a weightless file
(the converters synthesise 1 + ((i*k) % n) with the int wrap); a single
vertex; isolated vertices between rows.
"""
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "mst-artifact-sc23_b200"))
import ecl_mst as E  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "converters.npz")
TOOLS = {"pbbs": os.path.join(ROOT, "oracle", "_ref", "ecl2pbbs"),
         "mtx": os.path.join(ROOT, "oracle", "_ref", "ecl2mtx")}


def cases():
    rng = np.random.default_rng(7)
    g = E.gen_rmat(8, 8, 0.57, 0.19, 0.19, 11, 1 << 24)
    yield "rmat8", g.nindex, g.nlist, g.eweight
    w = rng.integers(-(2 ** 31), 2 ** 31, g.edges, dtype=np.int64).astype(np.int32)
    w[:4] = [2 ** 31 - 1, -(2 ** 31), 0, 2 ** 24 + 1]
    yield "rmat8_extreme", g.nindex, g.nlist, w
    h = E.gen_er(3000, 2.0, 5, 100)
    yield "er3000_weightless", h.nindex, h.nlist, None
    yield "single_vertex", np.zeros(2, np.int32), np.zeros(0, np.int32), np.zeros(0, np.int32)
    k = E.gen_grid(6, 9, 3, 1000)
    keep = np.ones(k.nodes, bool)
    keep[[0, 7, 8, 30]] = False  # drop every entry of a few vertices
    nl, ew, ni = [], [], [0]
    for v in range(k.nodes):
        for j in range(k.nindex[v], k.nindex[v + 1]):
            if keep[v] and keep[k.nlist[j]]:
                nl.append(k.nlist[j])
                ew.append(k.eweight[j])
        ni.append(len(nl))
    yield "grid_isolated", np.array(ni, np.int32), np.array(nl, np.int32), np.array(ew, np.int32)


def main():
    for t in TOOLS.values():
        if not os.path.exists(t):
            sys.exit(f"{t} missing: run `make -C oracle converters` where the reference sources exist")
    blobs, names = {}, []
    with tempfile.TemporaryDirectory() as tmp:
        for name, nindex, nlist, eweight in cases():
            names.append(name)
            g = E.Graph(nindex, nlist, eweight)
            path = os.path.join(tmp, name + ".egr")
            E.write_graph(g, path)
            blobs[f"{name}/nindex"] = g.nindex
            blobs[f"{name}/nlist"] = g.nlist
            blobs[f"{name}/eweight"] = np.zeros(0, np.int32) if eweight is None else g.eweight
            blobs[f"{name}/weightless"] = np.array(eweight is None)
            for fmt, tool in TOOLS.items():
                out = os.path.join(tmp, f"{name}.{fmt}")
                subprocess.run([tool, path, out], check=True, capture_output=True)
                with open(out, "rb") as f:
                    blobs[f"{name}/{fmt}"] = np.frombuffer(f.read(), np.uint8)
    np.savez_compressed(OUT, names=np.array(names), **blobs)
    print(f"wrote {OUT}: {len(names)} cases")


if __name__ == "__main__":
    main()
