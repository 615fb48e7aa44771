"""The oracle pinned against the reference itself (CPU only).

The oracle (oracle/kruskal.c) restates the reference's MST semantics; these
tests check it against (1) the committed golden fixtures, produced by the
reference's own cpuMST compiled from its sources, and (2) that compiled
reference directly, on generated graphs, when oracle/_ref is present.
"""
import numpy as np
import pytest

import ecl_mst as E
import oracle_lib as O


def test_oracle_matches_golden_inmst(golden):
    for name, c in golden.items():
        thr, filt = c["threshold"]
        got, w, fe = O.oracle_mst(c["nindex"], c["nlist"], c["eweight"], int(thr), int(filt))
        assert np.array_equal(got, c["inMST"]), name
        # the filtered two-phase order gives the same forest as plain Kruskal
        got2, w2, _ = O.oracle_mst(c["nindex"], c["nlist"], c["eweight"])
        assert np.array_equal(got2, c["inMST"]), name
        assert w == w2
        ref_w = int(c["eweight"][c["inMST"].astype(bool)].astype(np.int64).sum())
        assert w == ref_w % 2**64


def test_oracle_heuristic_matches_golden(golden):
    for name, c in golden.items():
        if len(c["nlist"]) == 0:
            continue
        n = len(c["nindex"]) - 1
        assert O.oracle_heuristic(n, c["eweight"]) == tuple(int(x) for x in c["threshold"]), name


def test_oracle_threshold_independent(golden):
    """For non-negative weights any threshold yields the same forest."""
    rng = np.random.default_rng(1)
    for name, c in golden.items():
        if len(c["nlist"]) == 0:
            continue
        for t in rng.choice(c["eweight"], 3):
            got, _, _ = O.oracle_mst(c["nindex"], c["nlist"], c["eweight"], int(t), 1)
            assert np.array_equal(got, c["inMST"]), (name, t)


def test_oracle_verify_counts(golden):
    c = golden["random_dense_3000"]
    ok, counts = O.oracle_verify(c["eweight"], c["inMST"], c["inMST"])
    assert ok and counts[2] == counts[3] == 0
    bad = c["inMST"].copy()
    j = int(np.flatnonzero(bad)[0])
    bad[j] = 0
    ok, counts = O.oracle_verify(c["eweight"], c["inMST"], bad)
    assert not ok and counts[2] == 1


@pytest.mark.skipif(not O.have_ref(), reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("family", ["grid", "rmat", "er", "rgg"])
def test_oracle_matches_reference_cpumst(family):
    if family == "grid":
        g = E.gen_grid(300, 300, 11, 1000)
    elif family == "rmat":
        g = E.gen_rmat(14, 16, 0.57, 0.19, 0.19, 12, 1 << 24)
    elif family == "er":
        g = E.gen_er(50000, 8, 13, 1 << 20)
    else:
        g = E.gen_rgg2d(50000, 3, 14, 1 << 20)
    t, f = O.oracle_heuristic(g.nodes, g.eweight)
    assert (t, f) == O.ref_threshold(g.nodes, g.eweight)
    ours, _, _ = O.oracle_mst(g.nindex, g.nlist, g.eweight, t, f)
    theirs = O.ref_cpu_mst(g.nindex, g.nlist, g.eweight)
    assert np.array_equal(ours, theirs)


def test_oracle_synth_matches_library():
    g = E.gen_rmat(12, 8, 0.57, 0.19, 0.19, 3, 100)
    w = O.oracle_synth(g.nindex, g.nlist)
    E.synthesize_weights(g)
    assert np.array_equal(w, g.eweight)
    assert (g.eweight >= 1).all()


def test_oracle_synth_wraps_like_int32():
    # i * k overflows int32 for these ids; the reference wraps and takes |.|
    n = 70000
    nindex = np.array([0] * 65537 + [1] * (n - 65536), np.int32)
    nindex[65537:] = 1
    nindex = np.zeros(n + 1, np.int32)
    nindex[65537:] = 1  # vertex 65536 has one entry
    nlist = np.array([69999], np.int32)
    w = O.oracle_synth(nindex, nlist)
    prod = np.int64(65536) * 69999
    wrapped = ((prod + 2**31) % 2**32) - 2**31
    r = int(np.fmod(wrapped, n))
    assert int(w[0]) == abs(1 + r)


@pytest.mark.parametrize("kind", ["rmat", "er", "grid"])
def test_oracle_generators_match_library(kind):
    """The oracle's input generators (oracle/graphgen.c, used by the
    benchmark's reference arm so that its process loads no product library)
    draw the same CSR as the library's generators, entry for entry."""
    import ecl_mst as E
    if kind == "rmat":
        want = E.gen_rmat(15, 16, 0.57, 0.19, 0.19, 2, 1 << 24)
        got = O.gen_rmat(15, 16, 0.57, 0.19, 0.19, 2, 1 << 24)
    elif kind == "er":
        want = E.gen_er(20_000, 8, 7, 1 << 20)
        got = O.gen_er(20_000, 8, 7, 1 << 20)
    else:
        want = E.gen_grid(123, 77, 1, 1_000_000)
        got = O.gen_grid(123, 77, 1, 1_000_000)
    for a, b in zip(got, (want.nindex, want.nlist, want.eweight)):
        assert np.array_equal(a, b)
