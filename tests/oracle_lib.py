"""ctypes access to the ORACLE (oracle/liboracle.so, oracle/_ref/libecl_ref.so).

Test infrastructure only: used as the checker by the tests, the smoke check
and the benchmark's CPU-baseline and reference legs. Nothing here loads the
product library, so a process that imports only this module (the
benchmark's reference arm) maps the oracle and the reference alone.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libecl_ref.so")

_orc = None
_ref = None


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def oracle():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle/liboracle.so missing: run `make -C oracle`")
        _orc = ctypes.CDLL(ORACLE_SO)
        _orc.oracle_mst.restype = ctypes.c_int
        _orc.oracle_mst.argtypes = [ctypes.c_int32, ctypes.c_int32] + [ctypes.c_void_p] * 3 + \
            [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
             ctypes.POINTER(ctypes.c_int64)]
        _orc.oracle_heuristic.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
        _orc.oracle_verify.restype = ctypes.c_int
        _orc.oracle_verify.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_int64)]
        _orc.oracle_synth.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _orc.gg_rmat.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(_GG)]
        _orc.gg_er.argtypes = [ctypes.c_int32, ctypes.c_double, ctypes.c_uint64, ctypes.c_int32,
                               ctypes.POINTER(_GG)]
        _orc.gg_grid.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_int32,
                                 ctypes.POINTER(_GG)]
        _orc.gg_free.argtypes = [ctypes.POINTER(_GG)]
    return _orc


class _GG(ctypes.Structure):
    _fields_ = [("nodes", ctypes.c_int32), ("edges", ctypes.c_int32), ("nindex", ctypes.c_void_p),
                ("nlist", ctypes.c_void_p), ("eweight", ctypes.c_void_p)]


def _take(fn, *args):
    g = _GG()
    st = fn(*args, ctypes.byref(g))
    if st != 0:
        raise RuntimeError(f"oracle generator failed ({st})")
    try:
        def arr(p, count):
            a = np.empty(count, np.int32)
            if count:
                ctypes.memmove(a.ctypes.data, p, 4 * count)
            return a
        return arr(g.nindex, g.nodes + 1), arr(g.nlist, g.edges), arr(g.eweight, g.edges)
    finally:
        oracle().gg_free(ctypes.byref(g))


def gen_rmat(scale, edge_factor, a, b, c, seed, wmax):
    """(nindex, nlist, eweight) of the seeded RMAT graph (oracle/graphgen.c)."""
    return _take(oracle().gg_rmat, scale, edge_factor, a, b, c, seed, wmax)


def gen_er(nodes, avg_degree, seed, wmax):
    return _take(oracle().gg_er, nodes, avg_degree, seed, wmax)


def gen_grid(rows, cols, seed, wmax):
    return _take(oracle().gg_grid, rows, cols, seed, wmax)


def have_ref():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        _ref = ctypes.CDLL(REF_SO)
        _ref.ref_cpu_mst.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 4
        _ref.ref_threshold.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        _ref.ref_gpu_mst.argtypes = [ctypes.c_int, ctypes.c_int] + [ctypes.c_void_p] * 3 + \
            [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]
    return _ref


def oracle_mst(nindex, nlist, eweight, threshold=0x7FFFFFFF, filtered=0):
    n, m = len(nindex) - 1, len(nlist)
    out = np.zeros(max(m, 1), np.uint8)
    w, fe = ctypes.c_uint64(), ctypes.c_int64()
    st = oracle().oracle_mst(n, m, _p(nindex), _p(nlist), _p(eweight), threshold, filtered, _p(out),
                             ctypes.byref(w), ctypes.byref(fe))
    assert st == 0
    return out[:m], w.value, fe.value


def oracle_heuristic(nodes, eweight):
    t, f = ctypes.c_int32(), ctypes.c_int32()
    oracle().oracle_heuristic(nodes, len(eweight), _p(eweight), ctypes.byref(t), ctypes.byref(f))
    return t.value, f.value


def oracle_verify(eweight, a, b):
    c = (ctypes.c_int64 * 4)()
    ok = oracle().oracle_verify(len(eweight), _p(eweight), _p(np.ascontiguousarray(a, np.uint8)),
                                _p(np.ascontiguousarray(b, np.uint8)), c)
    return bool(ok), list(c)


def oracle_synth(nindex, nlist):
    w = np.zeros(max(len(nlist), 1), np.int32)
    oracle().oracle_synth(len(nindex) - 1, _p(nindex), _p(nlist), _p(w))
    return w[: len(nlist)]


def ref_cpu_mst(nindex, nlist, eweight):
    n, m = len(nindex) - 1, len(nlist)
    out = np.zeros(max(m, 1), np.uint8)
    ref().ref_cpu_mst(n, m, _p(nindex), _p(nlist), _p(eweight), _p(out))
    return out[:m]


def ref_threshold(nodes, eweight):
    f, t = ctypes.c_int(), ctypes.c_int()
    ref().ref_threshold(nodes, len(eweight), _p(eweight), ctypes.byref(f), ctypes.byref(t))
    return t.value, f.value


def ref_gpu_mst(nindex, nlist, eweight, filtered, threshold):
    n, m = len(nindex) - 1, len(nlist)
    out = np.zeros(max(m, 1), np.uint8)
    sec = ctypes.c_double()
    ref().ref_gpu_mst(n, m, _p(nindex), _p(nlist), _p(eweight), filtered, threshold, _p(out),
                      ctypes.byref(sec))
    return out[:m], sec.value
