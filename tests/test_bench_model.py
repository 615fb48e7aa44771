"""The bench's algorithmic byte model (the roofline numerators), pinned to
hand-worked counts of the formulas it states: the round kernel per round
(first round in place; later rounds find, compact and reset) and the two
list-build scans. No GPU: the functions read a solve's stats dict."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

import bench  # noqa: E402


def _stats(wl, rounds, kept=(7, 5), filtered=1):
    return {"wl_real": wl, "rounds": rounds, "scan_kept": list(kept), "filtered": filtered}


def test_round_kernel_bytes_by_hand():
    n = 100
    st = _stats([[10, 8, 3], [20, 5]], [2, 1])
    # phase 0, round 0 (in place): read 16*10, guards 16*10; mark 16*8 + 16*8
    r00 = 160 + 160 + 128 + 128
    # phase 0, round 1: read 16*8, parent 8*8, guards 16*8, write 16*3, sparse reset 16*8 (4*8 < n);
    # mark 16*3 + 16*3
    r01 = 128 + 64 + 128 + 48 + 128 + 48 + 48
    # phase 1, round 0 (in place): 16*20 + 16*20; mark 16*5 + 16*5
    r10 = 320 + 320 + 80 + 80
    atomics = 2 * (8 + 3 + 5)  # the upper bound when the atomics were not counted
    assert bench.round_kernel_bytes(st, n) == r00 + r01 + r10 + 16 * atomics
    assert bench.round_kernel_bytes(st, n, atomics=4) == r00 + r01 + r10 + 16 * 4
    # a round holding at least n/4 entries clears the whole previous array (8n) instead
    dense = _stats([[10, 40, 3], [0]], [2, 0])
    base = 160 + 160 + 16 * 40 * 2
    later = 16 * 40 + 8 * 40 + 16 * 40 + 16 * 3 + 8 * n + 16 * 3 * 2
    assert bench.round_kernel_bytes(dense, n, atomics=0) == base + later


def test_scan_kernel_bytes_by_hand():
    n, m = 100, 1000
    light = 4 * (n + 1) + 8 * m + 20 * n + 16 * 7
    heavy = 8 * n + 4 * (n + 1) + 8 * m + 16 * 5
    assert bench.scan_kernel_bytes(_stats([[0], [0]], [0, 0]), n, m) == light + heavy
    assert bench.scan_kernel_bytes(_stats([[0], [0]], [0, 0], filtered=0), n, m) == light
