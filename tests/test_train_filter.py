"""Host logic of the learned schedule's training pipeline (train_filter.py):
the family and seed bookkeeping of saved sweep tables, the union of several
sweeps with per-sweep time weights, the soft labels and the decoding of a
network output into the sweep grid. No GPU: the sweep tables are synthetic."""
import os

import numpy as np
import pytest

import train_filter as TF


def _sweep(path, count, seed0=None, nmin=None, nmax=None, heur_scale=1.0, seed=0):
    rng = np.random.default_rng(seed)
    size = np.stack([rng.integers(10_000, 4_000_000, count), rng.integers(1 << 20, 1 << 27, count)], 1)
    tab = dict(x=rng.normal(0, 1, (count, 16)).astype(np.float32),
               times=rng.uniform(1, 2, (count, len(TF.QUANTILES), len(TF.SPLITS))).astype(np.float32),
               heur=(rng.uniform(1, 3, count) * heur_scale).astype(np.float32), size=size)
    kw = {}
    if seed0 is not None:
        kw["meta"] = np.array(dict(train_seed0=seed0 - 700_000, heldout_seed0=seed0, nmin=nmin, nmax=nmax),
                              dtype=object)
    np.savez_compressed(path, train_x=tab["x"], train_times=tab["times"], train_heur=tab["heur"],
                        train_size=tab["size"], heldout_x=tab["x"][:5], heldout_times=tab["times"][:5],
                        heldout_heur=tab["heur"][:5], heldout_size=tab["size"][:5], **kw)
    return tab


def test_dataset_without_record_is_the_first_sweep(tmp_path):
    p = os.path.join(tmp_path, "a.npz")
    _sweep(p, 20)
    tr, ho = TF.load_dataset(p)
    assert ho["seed"] == [TF.HELDOUT_SEED0 + i for i in range(5)]
    assert set(ho["nmin"]) == {10_000} and set(ho["nmax"]) == {4_000_000}
    assert ho["fam"] == [TF.family_of(s) for s in ho["seed"]]
    assert len(tr["x"]) == 20


def test_union_keeps_each_sweeps_seeds_and_weights(tmp_path):
    p1, p2 = os.path.join(tmp_path, "small.npz"), os.path.join(tmp_path, "large.npz")
    _sweep(p1, 30, seed=1)
    _sweep(p2, 10, seed0=950_000, nmin=4_000_000, nmax=33_554_432, heur_scale=50.0, seed=2)
    parts = [TF.load_dataset(p) for p in (p1, p2)]
    for t, _ in parts:
        t["rep"] = TF.time_weight(t)
    tr = TF.concat([t for t, _ in parts])
    ho = TF.concat([h for _, h in parts])
    assert tr["x"].shape == (40, 16) and len(tr["rep"]) == 40
    # each sweep is weighted against its own median: the 50x slower large
    # graphs do not all saturate at the maximum repeat count
    assert tr["rep"][30:].min() < 8 and tr["rep"].min() >= 1 and tr["rep"].max() <= 8
    assert TF.seed_ranges(ho) == [[900_000, 900_004, 10_000, 4_000_000], [950_000, 950_004, 4_000_000, 33_554_432]]
    assert ho["seed"][5:] == list(range(950_000, 950_005))


def test_label_prefers_the_fastest_setting():
    n, m = 1_000_000, 16_000_000
    times = np.full((len(TF.QUANTILES), len(TF.SPLITS)), 10.0, np.float32)
    qi, si = TF.QUANTILES.index(0.05), TF.SPLITS.index(16)
    times[qi, si] = 5.0
    lab = TF.label(times, n, m)
    assert abs(lab[0] - (np.log2(0.05) - TF.heuristic_log2_quantile(n, m))) < 1e-3
    assert abs(lab[1] - np.log2(16)) < 1e-3


@pytest.mark.parametrize("q,split", [(0.05, 4), (0.2, 8), (0.65, 16)])
def test_decoding_maps_the_label_back_to_its_grid_point(q, split):
    n, m = 2_000_000, 40_000_000
    pr = np.array([np.log2(q) - TF.heuristic_log2_quantile(n, m), np.log2(split)])
    qi, si = TF.predicted_setting(pr, n, m)
    assert TF.QUANTILES[qi] == q and TF.SPLITS[si] == split


def test_quantiles_above_the_no_filter_cut_run_unfiltered():
    n, m = 2_000_000, 40_000_000
    pr = np.array([np.log2(0.9) - TF.heuristic_log2_quantile(n, m), 3.0])
    qi, _ = TF.predicted_setting(pr, n, m)
    assert TF.QUANTILES[qi] == 1.0

