"""Training pipeline of the learned schedule (runs on a GPU).

1. Draw seeded training and held-out graphs on the device (the library's
   device generators) from the four families: 2D grid, Erdos-Renyi (average
   degree 8, 16 or 32), RMAT (.57, .19, .19; edge factor 8, 16 or 32) and
   random geometric 2D (average degree 3), vertex counts log-uniform in
   [--nmin, --nmax], weights uniform in [1, W] with W one of 2^20, 2^24, 2^30.
2. Label sweep: solve every graph with each of 16 filter quantiles x the 3
   distinct degree splits (the scans' entries per lane E = 4, 8, 16; larger
   splits select the same schedule) and keep the device times (best of
   --reps timed runs after one warm-up; repeated solves replay their captured
   CUDA graph). Every setting gives the same forest.
3. Label each graph with a soft minimum over the sweep (log2 quantile
   relative to the reference heuristic's, log2 split) and train the
   16 -> 64 -> 64 -> 2 MLP with the library's CUDA training kernel (Adam, one
   launch) on standardised features, graphs weighted by their solve time.
4. Evaluate on the held-out seeds: the sweep time at the predicted setting
   against the reference heuristic (its fallback and yardstick) and the best of
   the sweep, per family; then re-solve every held-out graph with the trained
   weights loaded, learned against heuristic, and report the measured gain
   and the share of graphs that are not slower.
5. Write the parameter blob (filter_weights.bin) and the JSON summary
   (filter_training.json) into --out-dir; with --dataset, also the sweep
   tables.

    python train_filter.py --train 3000 --heldout 500 --out-dir <dir> --dataset <sweeps.npz>
    python train_filter.py --eval-only <sweeps.npz> [<large.npz>] --weights <blob> --out-dir <dir>
    python train_filter.py --nmin 4000000 --nmax 33554432 --seed-offset 50000 \
        --train 500 --heldout 150 --out-dir <dir> --dataset <large.npz>
    python train_filter.py --from-datasets <sweeps.npz> <large.npz> --out-dir <dir>
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import ecl_mst as E  # noqa: E402

QUANTILES = [0.005, 0.01, 0.02, 0.03, 0.05, 0.07, 0.1, 0.15, 0.2, 0.3, 0.4, 0.5, 0.65, 0.8, 0.9, 1.0]
SPLITS = [4, 8, 16]  # degree splits selecting the scans' E = 4, 8, 16 entries per lane
FAMILIES = ["grid", "er", "rmat", "rgg"]
TRAIN_SEED0, HELDOUT_SEED0 = 200_000, 900_000


def family_of(seed):
    """Family name of seed `seed` (make_graph's first draw)."""
    return FAMILIES[int(np.random.default_rng(seed).integers(4))]


def make_graph(seed, nmin, nmax):
    """(DeviceGraph, family name) of training or held-out seed `seed`."""
    rng = np.random.default_rng(seed)
    fam = int(rng.integers(4))
    n = int(np.exp(rng.uniform(np.log(nmin), np.log(nmax))))
    wmax = int(rng.choice([1 << 20, 1 << 24, 1 << 30]))
    if fam == 0:
        r = max(2, int(np.sqrt(n)))
        return E.gen_grid_device(r, max(2, n // r), seed, wmax), "grid"
    if fam == 1:
        return E.gen_er_device(n, float(rng.choice([8, 16, 32])), seed, wmax), "er"
    if fam == 2:
        scale = max(10, int(round(np.log2(n))))
        ef = int(rng.choice([8, 16, 32]))
        ef = min(ef, (1 << 30) >> (scale + 1))  # at most 2^30 entries (edge factor 16 at scale 25)
        return E.gen_rmat_device(scale, ef, 0.57, 0.19, 0.19, seed, wmax), "rmat"
    return E.gen_rgg2d_device(n, 3.0, seed, wmax), "rgg"


def solve_ms(ctx, dg, out, opts, reps):
    """Best device time of `reps` timed solves after one warm-up."""
    best = 1e30
    for r in range(reps + 1):
        st = ctx.run_device(dg.nodes, dg.edges, dg.d_nindex, dg.d_nlist, dg.d_eweight, out.data_ptr(), opts=opts,
                            stats=True)
        if r > 0:
            best = min(best, st["ms_total"])
    return best


def sweep(ctx, dg, out, reps):
    feat = E.graph_features(dg.nodes, dg.edges, dg.d_nindex, dg.d_nlist, dg.d_eweight)
    times = np.zeros((len(QUANTILES), len(SPLITS)), np.float32)
    for qi, q in enumerate(QUANTILES):
        for si, sp in enumerate(SPLITS):
            times[qi, si] = solve_ms(ctx, dg, out, E.make_opts(mode=E.THRESH_QUANTILE, quantile=q, degree_split=sp),
                                     reps)
    heur = solve_ms(ctx, dg, out, E.make_opts(), reps)
    return feat, times, heur


def heuristic_log2_quantile(n, m):
    """log2 of the quantile the reference heuristic filters at (0 = no filter)."""
    if n < 1 or m // n < 4:
        return 0.0
    idx = min(19, int(3.0 * n * 20 / m))
    return float(np.log2((idx + 1) / 21.0))


def label(times, n, m, tau=0.03):
    """Soft label: softmin (temperature tau x best time) over the quantiles of
    the best split per quantile, as log2 q relative to the heuristic's, and
    the same over splits at the best quantile. Settings within a few percent
    of the best share the label instead of a noisy argmin picking one."""
    lq, ls = np.log2(QUANTILES), np.log2(SPLITS)
    tq = times.min(axis=1)
    w = np.exp(-(tq - tq.min()) / (tau * tq.min()))
    ts = times[int(np.argmin(tq))]
    ws = np.exp(-(ts - ts.min()) / (tau * ts.min()))
    return np.array([(w * lq).sum() / w.sum() - heuristic_log2_quantile(n, m), (ws * ls).sum() / ws.sum()],
                    np.float32)


NO_FILTER_LOG2Q = np.log2(0.8)  # as the device decodes: predicted quantiles above 0.8 run unfiltered


def predicted_setting(pr, n, m):
    """Grid point nearest the MLP's output (as the device applies it)."""
    lq = min(max(heuristic_log2_quantile(n, m) + float(pr[0]), -10.0), 0.0)
    q = 1.0 if lq >= NO_FILTER_LOG2Q else 2.0 ** lq
    sp = int(round(min(max(float(pr[1]), 1.0), 6.0)))
    qi = int(np.argmin([abs(np.log2(a) - np.log2(q)) for a in QUANTILES]))
    si = 0 if sp <= 2 else (1 if sp == 3 else 2)  # E = 4 for splits <= 4, 8 for 8, 16 above
    return qi, si


def collect(ctx, count, seed0, nmin, nmax, reps, torch):
    rows = []
    t0 = time.time()
    for i in range(count):
        dg, fam = make_graph(seed0 + i, nmin, nmax)
        out = torch.empty(max(dg.edges, 1), dtype=torch.uint8, device="cuda:0")
        f, tm, h = sweep(ctx, dg, out, reps)
        rows.append(dict(x=f, times=tm, heur=h, fam=fam, size=(dg.nodes, dg.edges)))
        dg.close()
        del out
        if (i + 1) % 100 == 0:
            print(f"  {i + 1}/{count} graphs swept, {time.time() - t0:.0f} s", flush=True)
    return dict(x=np.array([r["x"] for r in rows]), times=np.array([r["times"] for r in rows]),
                heur=np.array([r["heur"] for r in rows]), fam=[r["fam"] for r in rows],
                size=np.array([r["size"] for r in rows]))


def load_dataset(path):
    """Sweep tables of a dataset. Held-out graph i was drawn from seed
    heldout_seed0 + i with vertex counts in [nmin, nmax] (datasets without
    that record are the first sweep: seeds 900000.., 10^4..4*10^6)."""
    d = np.load(path, allow_pickle=True)
    tr = dict(x=d["train_x"], times=d["train_times"], heur=d["train_heur"], size=d["train_size"])
    ho = dict(x=d["heldout_x"], times=d["heldout_times"], heur=d["heldout_heur"], size=d["heldout_size"])
    meta = d["meta"].tolist() if "meta" in d.files else dict(heldout_seed0=HELDOUT_SEED0, nmin=10_000, nmax=4_000_000)
    k = len(ho["x"])
    ho["seed"] = [meta["heldout_seed0"] + i for i in range(k)]
    ho["nmin"] = [meta["nmin"]] * k
    ho["nmax"] = [meta["nmax"]] * k
    ho["fam"] = [family_of(sd) for sd in ho["seed"]]
    return tr, ho


def seed_ranges(ho):
    """[first seed, last seed, nmin, nmax] of each held-out sweep in `ho`."""
    r = {}
    for sd, lo, hi in zip(ho["seed"], ho["nmin"], ho["nmax"]):
        a, b = r.get((lo, hi), (sd, sd))
        r[(lo, hi)] = (min(a, sd), max(b, sd))
    return [[int(a), int(b), int(lo), int(hi)] for (lo, hi), (a, b) in sorted(r.items())]


def concat(parts):
    out = {}
    for key in parts[0]:
        vals = [p[key] for p in parts]
        out[key] = np.concatenate(vals) if isinstance(vals[0], np.ndarray) else sum((list(v) for v in vals), [])
    return out


def time_weight(tr):
    """Repeat count of each graph: its solve time over the sweep's median,
    1..8 (big graphs carry the time)."""
    return np.clip(np.round(tr["heur"] / np.median(tr["heur"])), 1, 8).astype(int)


def train_on(tr, seed, epochs, lr):
    """The MLP trained by the library's CUDA kernel on sweep tables."""
    x = tr["x"]
    mean, std = x.mean(0), x.std(0) + 1e-6
    y = np.stack([label(t, n, m) for t, (n, m) in zip(tr["times"], tr["size"])])
    rep = tr["rep"] if "rep" in tr else time_weight(tr)
    order = np.random.default_rng(seed).permutation(int(rep.sum()))
    xs = np.repeat((x - mean) / std, rep, 0)[order].astype(np.float32)
    ys = np.repeat(y, rep, 0)[order]
    p0 = E.mlp_init(seed, mean=mean, std=std)
    return E.mlp_train(p0, xs, ys, epochs=epochs, lr=lr)


def run(args):
    import torch
    summary_extra = {}
    parts = None
    if args.eval_only or args.from_datasets:
        parts = [load_dataset(d) for d in (args.from_datasets or args.eval_only)]
        args.nmin = min(min(h["nmin"]) for _, h in parts)
        args.nmax = max(max(h["nmax"]) for _, h in parts)
    # largest graphs drawn: RMAT scale 22 at edge factor 32 and ER n_max at degree
    # 32; with vertex counts up to 2^25, RMAT scale 25 at edge factor 16 and ER
    # 2^25 at degree 32 (about 1.07e9 entries)
    big = args.nmax > 4_200_000
    if big and args.nmax > 1 << 25:
        raise SystemExit("--nmax above 2^25 needs a larger context")
    ctx = E.Context(1 << 25, 1_100_000_000) if big else E.Context(1 << 23, 300_000_000)
    if parts:
        # saved sweep tables: train on their union (or take the shipped weights),
        # evaluate the current decoding, and measure the held-out graphs again
        for t, _ in parts:
            t["rep"] = time_weight(t)  # each sweep weighted against its own median
        tr = concat([t for t, _ in parts])
        ho = concat([h for _, h in parts])
        if args.eval_only:
            p = np.fromfile(args.weights, np.float32)
            hist = None
            summary_extra["evaluated"] = "the shipped weights on the saved held-out sweeps, and measured again"
        else:
            p, hist = train_on(tr, args.seed, args.epochs, args.lr)
            summary_extra["datasets"] = [os.path.basename(d) for d in args.from_datasets]
        if args.eval_only:
            summary_extra["datasets"] = [os.path.basename(d) for d in args.eval_only]
        args.train, args.heldout = len(tr["x"]), len(ho["x"])
    else:
        t0 = time.time()
        tr = collect(ctx, args.train, TRAIN_SEED0 + args.seed_offset, args.nmin, args.nmax, args.reps, torch)
        print(f"train: {args.train} graphs swept in {time.time() - t0:.0f} s", flush=True)
        t0 = time.time()
        h0 = HELDOUT_SEED0 + args.seed_offset
        ho = collect(ctx, args.heldout, h0, args.nmin, args.nmax, args.reps, torch)
        ho["seed"] = [h0 + i for i in range(args.heldout)]
        ho["nmin"], ho["nmax"] = [args.nmin] * args.heldout, [args.nmax] * args.heldout
        print(f"heldout: {args.heldout} graphs swept in {time.time() - t0:.0f} s", flush=True)
        p, hist = train_on(tr, args.seed, args.epochs, args.lr)

    # held-out, from the sweep tables: time at the predicted grid point
    pred = E.mlp_forward(p, ho["x"])
    res = []
    for pr, tm, h, (n, m) in zip(pred, ho["times"], ho["heur"], ho["size"]):
        qi, si = predicted_setting(pr, n, m)
        res.append((float(tm[qi, si]), float(h), float(tm.min())))
    res = np.array(res)
    fams = np.array(ho["fam"])
    gated = ho["size"][:, 1] >= (1 << 20)  # graphs the library runs the learned schedule on

    def gain(sel):
        return {"graphs": int(sel.sum()), "ms_learned": float(res[sel, 0].sum()),
                "ms_heuristic": float(res[sel, 1].sum()), "ms_best": float(res[sel, 2].sum()),
                "gain_over_heuristic": float(res[sel, 1].sum() / max(res[sel, 0].sum(), 1e-9)),
                "not_slower": float((res[sel, 0] <= res[sel, 1] * 1.02).mean()) if sel.any() else None}

    summary = {
        "train_graphs": args.train, "heldout_graphs": args.heldout, "nmin": args.nmin, "nmax": args.nmax,
        "heldout_seed_ranges": seed_ranges(ho),
        "quantiles": QUANTILES, "splits": SPLITS, "reps": args.reps, "epochs": args.epochs, "lr": args.lr,
        "loss_first": None if hist is None else float(hist[0]),
        "loss_last": None if hist is None else float(hist[-1]),
        "sweep_heldout": gain(np.ones(len(res), bool)),
        "sweep_heldout_by_family": {f: gain(fams == f) for f in FAMILIES},
        "sweep_heldout_learned_size": gain(gated),
        "no_filter_above_quantile": 0.8, "learned_min_edges": 1 << 20,
    }
    summary.update(summary_extra)

    # measured: re-solve the held-out graphs with the trained weights loaded
    E.learned_set_weights(p)
    meas = []
    for i in range(args.heldout):
        dg, fam = make_graph(ho["seed"][i], ho["nmin"][i], ho["nmax"][i])
        out = torch.empty(max(dg.edges, 1), dtype=torch.uint8, device="cuda:0")
        th = tl = 1e30
        for _ in range(2):  # interleaved, best of each
            th = min(th, solve_ms(ctx, dg, out, E.make_opts(mode=E.THRESH_HEURISTIC), args.reps))
            tl = min(tl, solve_ms(ctx, dg, out, E.make_opts(mode=E.THRESH_LEARNED), args.reps))
        meas.append((fam, dg.edges, th, tl))
        dg.close()
        del out
    ctx.close()

    def mgain(sel):
        th = sum(t for (f, m, t, _), s in zip(meas, sel) if s)
        tl = sum(t for (f, m, _, t), s in zip(meas, sel) if s)
        ns = [tl_ <= th_ * 1.02 for (f, m, th_, tl_), s in zip(meas, sel) if s]
        return {"graphs": int(sum(sel)), "ms_heuristic": th, "ms_learned": tl, "gain": th / max(tl, 1e-9),
                "not_slower": float(np.mean(ns)) if ns else None}

    big = [m >= (1 << 20) for (_, m, _, _) in meas]
    summary["measured_heldout"] = mgain([True] * len(meas))
    summary["measured_heldout_learned_size"] = mgain(big)
    summary["measured_heldout_by_family"] = {f: mgain([fm == f and b for (fm, _, _, _), b in zip(meas, big)])
                                             for f in FAMILIES}
    large = [n > 4_200_000 for n in ho["size"][:, 0]]
    if any(large):
        summary["measured_heldout_above_4M_vertices"] = mgain(large)
        summary["measured_heldout_above_4M_by_family"] = {
            f: mgain([fm == f and b for (fm, _, _, _), b in zip(meas, large)]) for f in FAMILIES}
    os.makedirs(args.out_dir, exist_ok=True)
    np.asarray(p, np.float32).tofile(os.path.join(args.out_dir, "filter_weights.bin"))
    if args.dataset and not (args.eval_only or args.from_datasets):
        meta = dict(train_seed0=TRAIN_SEED0 + args.seed_offset, heldout_seed0=HELDOUT_SEED0 + args.seed_offset,
                    nmin=args.nmin, nmax=args.nmax)
        np.savez_compressed(args.dataset, train_x=tr["x"], train_times=tr["times"], train_heur=tr["heur"],
                            train_size=tr["size"], heldout_x=ho["x"], heldout_times=ho["times"],
                            heldout_heur=ho["heur"], heldout_size=ho["size"], meta=np.array(meta, dtype=object))
    with open(os.path.join(args.out_dir, "filter_training.json"), "w") as f:
        json.dump(summary, f, indent=1)
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=2000)
    ap.add_argument("--heldout", type=int, default=500)
    ap.add_argument("--nmin", type=int, default=10_000)
    ap.add_argument("--nmax", type=int, default=4_000_000)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out-dir", default=HERE)
    ap.add_argument("--dataset", default=None, help="also write the sweep tables (.npz) here")
    ap.add_argument("--eval-only", nargs="+", default=None, metavar="DATASET",
                    help="evaluate --weights on these saved sweep tables and measure the held-out graphs again")
    ap.add_argument("--weights", default=os.path.join(HERE, "filter_weights.bin"))
    ap.add_argument("--from-datasets", nargs="+", default=None, metavar="DATASET",
                    help="train on the union of these saved sweep tables instead of sweeping")
    ap.add_argument("--seed-offset", type=int, default=0,
                    help="added to the training and held-out seed ranges (a second, disjoint sweep)")
    run(ap.parse_args())
