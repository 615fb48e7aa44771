"""Runtime and throughput tables from ecl_mst command-line output.

Restates the median / throughput computation of the artifact's table
scripts (generate_compare_tables.py:39-63, generate_deoptimize_tables.py) for
the output of this library's `ecl_mst` binary, which prints the same blocks
as the reference binary: a line "input: <graph path>" followed by one
runtime line per run (seconds). Per input and output file the table holds
the median runtime and the throughput in Medges/s = directed CSR entries /
median runtime / 1e6. The entry counts come from a {input name: edges}
mapping (the reference hard-codes one, generate_compare_tables.py:16-33) or,
when the graph file named on the "input:" line exists, from its ECLgraph
header (int32 nodes, int32 edges; ECLgraph.h:37-50).

    python compare_tables.py ecl_mst_out.csv ecl_mst_NAG_out.csv \
        [--sizes sizes.json] [--prefix comparison]

writes <prefix>_runtimes.csv and <prefix>_throughputs.csv in the reference's
layout: a header row of output names, then one row per input.
"""
import argparse
import json
import os
import statistics
import struct


def parse_runs(text):
    """[(input path, [runtimes...]), ...] from one output file's text."""
    blocks, cur = [], None
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("input:"):
            cur = (line[len("input:"):].strip(), [])
            blocks.append(cur)
            continue
        if cur is None or not line:
            continue
        try:
            cur[1].append(float(line))
        except ValueError:
            cur = None  # a trailer line ("forest: ...") ends the block
    return blocks


def input_name(path):
    """The reference's input key: the file name without directory and .egr."""
    base = os.path.basename(path)
    return base[:-4] if base.endswith(".egr") else base


def edges_of(path, sizes):
    name = input_name(path)
    if name in sizes:
        return sizes[name]
    if os.path.exists(path):
        with open(path, "rb") as f:
            _, edges = struct.unpack("<ii", f.read(8))
        return edges
    raise KeyError(f"no entry count for {name}: give --sizes or keep the graph file")


def tables(outputs, sizes=None, runs=None):
    """outputs: {output name: file text}. Returns (inputs, names, runtime, throughput)
    where runtime[i][k] / throughput[i][k] belong to input i and output k (None when an
    output lacks that input). `runs` keeps only the first `runs` values of a block, as the
    reference reads exactly 9 (generate_compare_tables.py:50-53)."""
    sizes = sizes or {}
    names = list(outputs)
    parsed = {k: parse_runs(v) for k, v in outputs.items()}
    inputs = []
    for k in names:
        for path, _ in parsed[k]:
            if input_name(path) not in [input_name(p) for p in inputs]:
                inputs.append(path)
    runtime = [[None] * len(names) for _ in inputs]
    throughput = [[None] * len(names) for _ in inputs]
    for c, k in enumerate(names):
        for path, vals in parsed[k]:
            if runs:
                vals = vals[:runs]
            if not vals:
                continue
            r = next(i for i, p in enumerate(inputs) if input_name(p) == input_name(path))
            med = statistics.median(vals)
            runtime[r][c] = med
            throughput[r][c] = edges_of(path, sizes) / med / 1e6
    return inputs, names, runtime, throughput


def write_csv(path, inputs, names, table):
    with open(path, "w") as w:
        w.write("," + "".join(n.replace("_out.csv", "") + ", " for n in names))
        for i, p in enumerate(inputs):
            w.write("\n" + input_name(p))
            for v in table[i]:
                w.write("," + ("" if v is None else str(v)))


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("outputs", nargs="+", help="ecl_mst output files")
    ap.add_argument("--sizes", help="JSON {input name: directed CSR entries}")
    ap.add_argument("--runs", type=int, default=9, help="runtime lines per block to use")
    ap.add_argument("--prefix", default="comparison")
    args = ap.parse_args()
    sizes = json.load(open(args.sizes)) if args.sizes else {}
    outs = {os.path.basename(p): open(p).read() for p in args.outputs}
    inputs, names, rt, tp = tables(outs, sizes, args.runs)
    write_csv(f"{args.prefix}_runtimes.csv", inputs, names, rt)
    write_csv(f"{args.prefix}_throughputs.csv", inputs, names, tp)
    print(f"wrote {args.prefix}_runtimes.csv and {args.prefix}_throughputs.csv")


if __name__ == "__main__":
    main()
