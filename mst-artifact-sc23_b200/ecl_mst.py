"""Python binding of the ecl_mst C ABI (include/ecl_mst.h) via ctypes.

It mirrors the reference's interface for this path (alexfallin/MST-Artifact-SC23):
  - ``Graph``: the ECLgraph struct (ECL-MST/ECLgraph.h:29-35) as numpy arrays;
  - ``read_graph`` / ``write_graph``: readECLgraph / writeECLgraph (ECLgraph.h:37-80);
  - ``mst``: gpuMST<filter> plus main's threshold choice (ECL_MST.cu:265-362, :432-444),
    returning the per-CSR-entry ``inMST`` flags (uint8, edges long);
  - ``verify``: verify() (ECL_MST.cu:365-386).

There is no fallback: if ``libecl_mst.so`` (built by ``make`` in this directory)
is missing, ``load()`` raises. Errors from the library come back as
``EclError`` with the library's status code (the reference would exit(-1)).
"""
import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint64, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("ECL_MST_LIB") or os.path.join(_HERE, "libecl_mst.so")

ECL_OK = 0
STATUS = {
    0: "ok", -1: "invalid argument", -2: "i/o error", -3: "malformed graph",
    -4: "allocation failed", -5: "CUDA error", -6: "no CUDA device",
    -7: "capacity exceeded", -8: "device wait limit reached",
    -9: "input exceeds the supported maximum", -10: "unsupported option",
}
THRESH_HEURISTIC, THRESH_NONE, THRESH_EXPLICIT, THRESH_QUANTILE, THRESH_LEARNED = range(5)
FLAG_L2_PERSIST, FLAG_STATS, FLAG_NO_SMALL_TAIL = 1, 2, 4
# ablation switches (the answer is unchanged; see include/ecl_mst.h)
FLAG_NO_GUARDS, FLAG_NO_WARP_COOP, FLAG_DEDUP, FLAG_NO_FIND_CACHE = 8, 16, 32, 64
# direct launches instead of replaying a captured solve (keeps per-phase timings)
FLAG_NO_GRAPH = 128
# the reference's later deoptimization steps (single-graph contexts only)
FLAG_NO_IMPLICIT_COMPRESSION, FLAG_NO_TUPLES, FLAG_NO_DATA_DRIVEN, FLAG_NO_EDGE_BASED = 256, 512, 1024, 2048
MAX_ROUNDS = 64


class EclError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"{what}: {STATUS.get(status, 'unknown')} ({status})")


class EclGraphC(ctypes.Structure):
    _fields_ = [("nodes", c_int32), ("edges", c_int32), ("nindex", c_void_p),
                ("nlist", c_void_p), ("eweight", c_void_p)]


class MstOpts(ctypes.Structure):
    _fields_ = [("threshold_mode", c_int32), ("threshold", c_int32), ("quantile", c_float),
                ("degree_split", c_int32), ("round_min_tiles", c_int32), ("ctas_per_sm", c_int32),
                ("small_tail", c_int32), ("flags", c_int32), ("batch_small_edges", c_int32),
                ("batch_large_streams", c_int32), ("reserved", c_int32 * 6)]


class MstStats(ctypes.Structure):
    _fields_ = [("threshold", c_int32), ("filtered", c_int32), ("degree_split", c_int32),
                ("rounds", c_int32 * 2), ("status", c_int32), ("scan_kept", c_int64 * 2),
                ("wl_in", (c_int64 * MAX_ROUNDS) * 2), ("atomics", c_int64),
                ("forest_edges", c_int64), ("forest_weight", c_uint64),
                ("ms_total", c_float), ("ms_rounds", c_float), ("ms_scan", c_float),
                ("us_scan", (c_float * 3) * 2), ("us_round", ((c_float * 2) * MAX_ROUNDS) * 2),
                ("wl_real", (c_int64 * MAX_ROUNDS) * 2)]

    def as_dict(self):
        return {
            "threshold": self.threshold, "filtered": self.filtered,
            "degree_split": self.degree_split, "rounds": list(self.rounds),
            "status": self.status, "scan_kept": list(self.scan_kept),
            "wl_in": [[int(x) for x in self.wl_in[p][: max(self.rounds[p], 0) + 1]] for p in range(2)],
            "wl_real": [[int(x) for x in self.wl_real[p][: max(self.rounds[p], 0) + 1]] for p in range(2)],
            "atomics": self.atomics, "forest_edges": self.forest_edges,
            "forest_weight": self.forest_weight, "ms_total": self.ms_total,
            "ms_rounds": self.ms_rounds, "ms_scan": self.ms_scan,
            "us_scan": [list(self.us_scan[p]) for p in range(2)],
            "us_round": [[list(self.us_round[p][r]) for r in range(max(self.rounds[p], 0))] for p in range(2)],
        }


class EclBatchC(ctypes.Structure):
    _fields_ = [("num_graphs", c_int32), ("nodes", c_void_p), ("edges", c_void_p), ("nindex_off", c_void_p),
                ("edge_off", c_void_p), ("nindex", c_void_p), ("nlist", c_void_p), ("eweight", c_void_p)]


class BatchStats(ctypes.Structure):
    _fields_ = [("graphs_small", c_int32), ("graphs_large", c_int32), ("status", c_int32),
                ("graph_replay", c_int32), ("edges_total", c_int64), ("ms_total", c_float),
                ("ms_small", c_float), ("ms_large", c_float)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None


def load():
    """Load libecl_mst.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: run `make` in {_HERE} (no CPU fallback exists)")
    lib = ctypes.CDLL(LIB_PATH)
    G = POINTER(EclGraphC)
    sig = {
        "ecl_status_string": (c_char_p, [c_int]),
        "ecl_version": (c_char_p, []),
        "ecl_read_graph": (c_int, [c_char_p, G]),
        "ecl_write_graph": (c_int, [G, c_char_p]),
        "ecl_free_graph": (None, [G]),
        "ecl_synthesize_weights": (c_int, [G]),
        "ecl_validate_graph": (c_int, [G]),
        "ecl_gen_grid": (c_int, [c_int32, c_int32, c_uint64, c_int32, c_int, G]),
        "ecl_gen_er": (c_int, [c_int32, c_double, c_uint64, c_int32, c_int, G]),
        "ecl_gen_rmat": (c_int, [c_int32, c_int32, c_double, c_double, c_double, c_uint64, c_int32, c_int, G]),
        "ecl_gen_rgg2d": (c_int, [c_int32, c_double, c_uint64, c_int32, c_int, G]),
        "ecl_gen_batch_graph": (c_int, [c_int32, c_uint64, c_int32, c_int32, c_int32, G, POINTER(c_int32)]),
        "ecl_heuristic_threshold": (c_int, [G, POINTER(c_int32), POINTER(c_int32)]),
        "ecl_default_opts": (None, [POINTER(MstOpts)]),
        "ecl_mst_run": (c_int, [G, c_void_p, POINTER(MstOpts), POINTER(MstStats)]),
        "ecl_mst_ctx_create": (c_int, [c_int, c_int64, c_int64, POINTER(c_void_p)]),
        "ecl_mst_ctx_destroy": (None, [c_void_p]),
        "ecl_mst_ctx_run_host": (c_int, [c_void_p, G, c_void_p, POINTER(MstOpts), POINTER(MstStats)]),
        "ecl_mst_run_device": (c_int, [c_void_p, G, c_void_p, POINTER(MstOpts), c_void_p, POINTER(MstStats)]),
        "ecl_mst_ctx_sync": (c_int, [c_void_p]),
        "ecl_mst_run_device_noalloc": (c_int, [G, c_void_p, POINTER(MstOpts), c_void_p]),
        "ecl_mst_ctx_stream": (c_void_p, [c_void_p]),
        "ecl_mst_ctx_l2_reset": (c_int, [c_void_p]),
        "ecl_mst_ctx_learned_features": (c_int, [c_void_p, c_void_p]),
        "ecl_mst_ctx_run_host_async": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
        "ecl_mst_ctx_wait": (c_int, [c_void_p]),
        "ecl_host_alloc_pinned": (c_int, [ctypes.c_size_t, POINTER(c_void_p)]),
        "ecl_host_free_pinned": (None, [c_void_p]),
        "ecl_batch_ctx_create": (c_int, [c_int, c_int32, c_int64, c_int64, c_int32, POINTER(c_void_p)]),
        "ecl_batch_ctx_destroy": (None, [c_void_p]),
        "ecl_mst_run_batch_device": (c_int, [c_void_p, POINTER(EclBatchC), c_void_p, POINTER(MstOpts), c_void_p,
                                             POINTER(BatchStats)]),
        "ecl_batch_autotune": (c_int, [c_void_p, POINTER(EclBatchC), c_void_p, POINTER(MstOpts), POINTER(MstOpts),
                                       POINTER(c_float)]),
        "ecl_learned_set_weights": (c_int, [c_void_p, c_int]),
        "ecl_learned_has_weights": (c_int, []),
        "ecl_graph_features": (c_int, [G, c_void_p]),
        "ecl_mlp_forward": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
        "ecl_mlp_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, POINTER(c_float)]),
        "ecl_mlp_train": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_float, c_void_p]),
        "ecl_verify": (c_int, [G, c_void_p, c_void_p, POINTER(c_int64), POINTER(c_uint64), POINTER(c_uint64)]),
        "ecl_csr_from_pairs_device": (c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_int32, c_uint64,
                                              c_int32, c_void_p, G]),
        "ecl_gen_grid_device": (c_int, [c_int32, c_int32, c_uint64, c_int32, c_void_p, G]),
        "ecl_gen_er_device": (c_int, [c_int32, c_double, c_uint64, c_int32, c_void_p, G]),
        "ecl_gen_rmat_device": (c_int, [c_int32, c_int32, c_double, c_double, c_double, c_uint64, c_int32,
                                        c_void_p, G]),
        "ecl_gen_rgg2d_device": (c_int, [c_int32, c_double, c_uint64, c_int32, c_void_p, G]),
        "ecl_gen_batch_graph_device": (c_int, [c_int32, c_uint64, c_int32, c_int32, c_int32, c_void_p, G,
                                               POINTER(c_int32)]),
        "ecl_free_device_graph": (None, [G]),
        "ecl_graph_to_host": (c_int, [G, G]),
        "ecl_gen_batch_device": (c_int, [c_int32, c_uint64, c_int32, c_int32, c_int32, c_int32, c_void_p,
                                         POINTER(EclBatchC), c_void_p]),
        "ecl_free_device_batch": (None, [POINTER(EclBatchC)]),
        "ecl_write_pbbs": (c_int, [G, c_char_p]),
        "ecl_write_mtx": (c_int, [G, c_char_p]),
        "ecl_forest_weight": (c_uint64, [G, c_void_p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status, what):
    if status != ECL_OK:
        raise EclError(status, what)


def _ptr(a):
    return None if a is None else a.ctypes.data_as(c_void_p)


class Graph:
    """ECLgraph: int32 CSR (nindex[nodes+1], nlist[edges], optional eweight[edges])."""

    def __init__(self, nindex, nlist, eweight=None):
        self.nindex = np.ascontiguousarray(nindex, dtype=np.int32)
        self.nlist = np.ascontiguousarray(nlist, dtype=np.int32)
        self.eweight = None if eweight is None else np.ascontiguousarray(eweight, dtype=np.int32)
        self.nodes = int(self.nindex.shape[0]) - 1
        self.edges = int(self.nlist.shape[0])

    def struct(self):
        return EclGraphC(self.nodes, self.edges, _ptr(self.nindex), _ptr(self.nlist), _ptr(self.eweight))

    @classmethod
    def _from_c(cls, gc):
        lib = load()
        n, m = gc.nodes, gc.edges
        nindex = np.ctypeslib.as_array(ctypes.cast(gc.nindex, POINTER(c_int32)), (n + 1,)).copy()
        if m > 0:
            nlist = np.ctypeslib.as_array(ctypes.cast(gc.nlist, POINTER(c_int32)), (m,)).copy()
            ew = (np.ctypeslib.as_array(ctypes.cast(gc.eweight, POINTER(c_int32)), (m,)).copy()
                  if gc.eweight else None)
        else:
            nlist = np.zeros(0, np.int32)
            ew = np.zeros(0, np.int32) if gc.eweight else None
        lib.ecl_free_graph(ctypes.byref(gc))
        return cls(nindex, nlist, ew)


def read_graph(path):
    gc = EclGraphC()
    _check(load().ecl_read_graph(os.fsencode(path), ctypes.byref(gc)), f"read {path}")
    return Graph._from_c(gc)


def write_graph(g, path):
    gs = g.struct()
    _check(load().ecl_write_graph(ctypes.byref(gs), os.fsencode(path)), f"write {path}")


def synthesize_weights(g):
    """Fill g.eweight with the reference's synthetic weights (ECL_MST.cu:410-419)."""
    g.eweight = np.zeros(g.edges, np.int32)
    gs = g.struct()
    _check(load().ecl_synthesize_weights(ctypes.byref(gs)), "synthesize_weights")
    return g


def validate_graph(g):
    gs = g.struct()
    return load().ecl_validate_graph(ctypes.byref(gs))


def gen_grid(rows, cols, seed, wmax, threads=0):
    gc = EclGraphC()
    _check(load().ecl_gen_grid(rows, cols, seed, wmax, threads, ctypes.byref(gc)), "gen_grid")
    return Graph._from_c(gc)


def gen_er(nodes, avg_degree, seed, wmax, threads=0):
    gc = EclGraphC()
    _check(load().ecl_gen_er(nodes, avg_degree, seed, wmax, threads, ctypes.byref(gc)), "gen_er")
    return Graph._from_c(gc)


def gen_rmat(scale, edge_factor, a, b, c, seed, wmax, threads=0):
    gc = EclGraphC()
    _check(load().ecl_gen_rmat(scale, edge_factor, a, b, c, seed, wmax, threads, ctypes.byref(gc)), "gen_rmat")
    return Graph._from_c(gc)


def gen_rgg2d(nodes, avg_degree, seed, wmax, threads=0):
    gc = EclGraphC()
    _check(load().ecl_gen_rgg2d(nodes, avg_degree, seed, wmax, threads, ctypes.byref(gc)), "gen_rgg2d")
    return Graph._from_c(gc)


def gen_batch_graph(index, seed0=1000, nmin=1000, nmax=2_000_000, wmax=1 << 20):
    """Graph `index` of the mixed-family batch; returns (Graph, family 0..3)."""
    gc = EclGraphC()
    fam = c_int32()
    _check(load().ecl_gen_batch_graph(index, seed0, nmin, nmax, wmax, ctypes.byref(gc), ctypes.byref(fam)),
           "gen_batch_graph")
    return Graph._from_c(gc), fam.value


def gen_batch(count, seed0=1000, nmin=1000, nmax=2_000_000, wmax=1 << 20, threads=0):
    """The first `count` graphs of the mixed batch, generated in parallel."""
    from concurrent.futures import ThreadPoolExecutor
    workers = threads or os.cpu_count() or 1
    with ThreadPoolExecutor(workers) as ex:
        return list(ex.map(lambda i: gen_batch_graph(i, seed0, nmin, nmax, wmax)[0], range(count)))


def write_pbbs(g, path):
    """PBBS WeightedEdgeArray text, as PBBS_CPU/inputs/ecl2pbbs_genweights.cpp writes it."""
    gs = g.struct()
    _check(load().ecl_write_pbbs(ctypes.byref(gs), os.fsencode(path)), f"write_pbbs {path}")


def write_mtx(g, path):
    """MatrixMarket text, as cuGraph_GPU/inputs/ecl2mtx_genweights_cugraph.cpp writes it."""
    gs = g.struct()
    _check(load().ecl_write_mtx(ctypes.byref(gs), os.fsencode(path)), f"write_mtx {path}")


# ------------------------------------------------------ GPU-side preprocessing
WEIGHTS_GIVEN, WEIGHTS_HASH, WEIGHTS_SYNTH = 0, 1, 2


class DeviceGraph:
    """An ECLgraph whose arrays live in device memory (cudaMalloc'd by the
    library); ``to_host()`` copies it into a ``Graph``."""

    def __init__(self, gc):
        self._lib = load()
        self.c = gc
        self.nodes, self.edges = gc.nodes, gc.edges

    @property
    def d_nindex(self):
        return self.c.nindex

    @property
    def d_nlist(self):
        return self.c.nlist

    @property
    def d_eweight(self):
        return self.c.eweight

    def to_host(self):
        h = EclGraphC()
        _check(self._lib.ecl_graph_to_host(ctypes.byref(self.c), ctypes.byref(h)), "graph_to_host")
        return Graph._from_c(h)

    def close(self):
        if self.c.nindex:
            self._lib.ecl_free_device_graph(ctypes.byref(self.c))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_graph(fn, what, *args):
    gc = EclGraphC()
    _check(fn(*args, ctypes.byref(gc)), what)
    return DeviceGraph(gc)


def csr_from_pairs_device(nodes, pairs, d_u, d_v, d_w=None, rule=WEIGHTS_HASH, seed=0, wmax=1, stream=None):
    """Symmetric deduplicated CSR from `pairs` device-resident undirected pairs."""
    return _device_graph(load().ecl_csr_from_pairs_device, "csr_from_pairs_device", nodes, pairs, d_u, d_v, d_w,
                         rule, seed, wmax, stream)


def gen_grid_device(rows, cols, seed, wmax, stream=None):
    return _device_graph(load().ecl_gen_grid_device, "gen_grid_device", rows, cols, seed, wmax, stream)


def gen_er_device(nodes, avg_degree, seed, wmax, stream=None):
    return _device_graph(load().ecl_gen_er_device, "gen_er_device", nodes, avg_degree, seed, wmax, stream)


def gen_rmat_device(scale, edge_factor, a, b, c, seed, wmax, stream=None):
    return _device_graph(load().ecl_gen_rmat_device, "gen_rmat_device", scale, edge_factor, a, b, c, seed, wmax,
                         stream)


def gen_rgg2d_device(nodes, avg_degree, seed, wmax, stream=None):
    return _device_graph(load().ecl_gen_rgg2d_device, "gen_rgg2d_device", nodes, avg_degree, seed, wmax, stream)


def gen_batch_graph_device(index, seed0=1000, nmin=1000, nmax=2_000_000, wmax=1 << 20, stream=None):
    """Graph `index` of the mixed batch drawn on the device: (DeviceGraph, family)."""
    gc = EclGraphC()
    fam = c_int32()
    _check(load().ecl_gen_batch_graph_device(index, seed0, nmin, nmax, wmax, stream, ctypes.byref(gc),
                                             ctypes.byref(fam)), "gen_batch_graph_device")
    return DeviceGraph(gc), fam.value


class DeviceBatch:
    """The first `count` graphs of the mixed batch, drawn on the device and
    packed into one batch layout (ecl_gen_batch_device). Same interface as
    ``Batch`` for ``BatchContext``; the arrays stay on the device."""

    def __init__(self, count, seed0=1000, nmin=1000, nmax=2_000_000, wmax=1 << 20, align=4, stream=None):
        self._lib = load()
        self.c = EclBatchC()
        fam = np.zeros(count, np.int32)
        _check(self._lib.ecl_gen_batch_device(count, seed0, nmin, nmax, wmax, align, stream, ctypes.byref(self.c),
                                              _ptr(fam)), "gen_batch_device")
        self.family = fam
        self.num_graphs = count

        def arr(p, ct, dt):
            return np.ctypeslib.as_array(ctypes.cast(p, POINTER(ct)), (count,)).astype(dt)

        self.nodes = arr(self.c.nodes, c_int32, np.int32)
        self.edges = arr(self.c.edges, c_int32, np.int32)
        self.nindex_off = arr(self.c.nindex_off, c_int64, np.int64)
        self.edge_off = arr(self.c.edge_off, c_int64, np.int64)
        self.total_nindex = int(self.nindex_off[-1]) + -(-(int(self.nodes[-1]) + 1) // align) * align
        self.total_edges = int(self.edge_off[-1]) + -(-max(int(self.edges[-1]), 1) // align) * align
        self.d_nindex, self.d_nlist, self.d_eweight = self.c.nindex, self.c.nlist, self.c.eweight

    def struct(self, d_nindex=None, d_nlist=None, d_eweight=None):
        return EclBatchC(self.num_graphs, self.c.nodes, self.c.edges, self.c.nindex_off, self.c.edge_off,
                         d_nindex or self.d_nindex, d_nlist or self.d_nlist, d_eweight or self.d_eweight)

    def slice(self, inmst, g):
        a = int(self.edge_off[g])
        return inmst[a:a + int(self.edges[g])]

    def graph(self, g):
        """Host copy of graph g."""
        gc = EclGraphC(int(self.nodes[g]), int(self.edges[g]), self.d_nindex + 4 * int(self.nindex_off[g]),
                       self.d_nlist + 4 * int(self.edge_off[g]), self.d_eweight + 4 * int(self.edge_off[g]))
        h = EclGraphC()
        _check(self._lib.ecl_graph_to_host(ctypes.byref(gc), ctypes.byref(h)), "graph_to_host")
        return Graph._from_c(h)

    def select(self, idx):
        """A view of graphs `idx` of this batch (see ``BatchView``)."""
        return BatchView(self, idx)

    def close(self):
        if self.c.nindex:
            self._lib.ecl_free_device_batch(ctypes.byref(self.c))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def heuristic_threshold(g):
    """(threshold, filtered) of the reference rule (ECL_MST.cu:408,432-440)."""
    t, f = c_int32(), c_int32()
    gs = g.struct()
    _check(load().ecl_heuristic_threshold(ctypes.byref(gs), ctypes.byref(t), ctypes.byref(f)), "heuristic")
    return t.value, f.value


def make_opts(mode=THRESH_HEURISTIC, threshold=0, quantile=1.0, degree_split=0, small_tail=0, flags=0,
              round_min_tiles=0, ctas_per_sm=0, batch_large_streams=0):
    o = MstOpts()
    load().ecl_default_opts(ctypes.byref(o))
    o.threshold_mode = mode
    o.threshold = threshold
    o.quantile = quantile
    o.degree_split = degree_split
    o.small_tail = small_tail
    o.flags = flags
    o.round_min_tiles = round_min_tiles
    o.ctas_per_sm = ctas_per_sm
    o.batch_large_streams = batch_large_streams
    return o


def mst(g, opts=None):
    """One-shot solve (ecl_mst_run): returns (inMST uint8[edges], stats dict)."""
    out = np.zeros(max(g.edges, 1), np.uint8)
    st = MstStats()
    gs = g.struct()
    _check(load().ecl_mst_run(ctypes.byref(gs), _ptr(out), None if opts is None else ctypes.byref(opts),
                              ctypes.byref(st)), "ecl_mst_run")
    return out[: g.edges], st.as_dict()


def run_device_noalloc(nodes, edges, d_nindex, d_nlist, d_eweight, d_inMST, opts=None, stream=None):
    """Allocation-free solve (ecl_mst_run_device_noalloc): device pointers in
    and out, scratch in the library's static device array; returns after the
    solve. For callers that cannot allocate device memory."""
    gs = EclGraphC(nodes, edges, d_nindex, d_nlist, d_eweight)
    _check(load().ecl_mst_run_device_noalloc(ctypes.byref(gs), d_inMST,
                                             None if opts is None else ctypes.byref(opts), stream),
           "run_device_noalloc")


def verify(g, a, b):
    """verify() of the reference: (agree, counts[4], weight_a, weight_b)."""
    counts = (c_int64 * 4)()
    wa, wb = c_uint64(), c_uint64()
    gs = g.struct()
    a = np.ascontiguousarray(a, np.uint8)
    b = np.ascontiguousarray(b, np.uint8)
    ok = load().ecl_verify(ctypes.byref(gs), _ptr(a), _ptr(b), counts, ctypes.byref(wa), ctypes.byref(wb))
    return bool(ok), list(counts), wa.value, wb.value


class Context:
    """Reusable device workspace (ecl_mst_ctx)."""

    def __init__(self, max_nodes, max_edges, device=0):
        self._lib = load()
        h = c_void_p()
        _check(self._lib.ecl_mst_ctx_create(device, max_nodes, max_edges, ctypes.byref(h)), "ctx_create")
        self.handle = h
        self._inflight = []  # arrays of run_host_async calls not yet waited for

    def close(self):
        if self.handle:
            self._lib.ecl_mst_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream(self):
        return self._lib.ecl_mst_ctx_stream(self.handle)

    def run_host(self, g, opts=None, out=None, stats=True):
        """Host CSR in, host inMST out (H2D + solve + D2H)."""
        if out is None:
            out = np.zeros(max(g.edges, 1), np.uint8)
        st = MstStats() if stats else None
        gs = g.struct()
        _check(self._lib.ecl_mst_ctx_run_host(self.handle, ctypes.byref(gs), _ptr(out),
                                              None if opts is None else ctypes.byref(opts),
                                              None if st is None else ctypes.byref(st)), "ctx_run_host")
        return out[: g.edges], (st.as_dict() if st is not None else None)

    def run_host_async(self, g, opts=None, out=None):
        """Enqueue a host-buffer solve (copy in, solve, copy back) that overlaps
        the previous one; the result lands in `out` by the next wait(). The
        arrays are kept referenced until then."""
        if out is None:
            out = np.zeros(max(g.edges, 1), np.uint8)
        gs = g.struct()
        keep = (g, out, gs, opts)
        _check(self._lib.ecl_mst_ctx_run_host_async(self.handle, ctypes.byref(gs), _ptr(out),
                                                    None if opts is None else ctypes.byref(opts)),
               "ctx_run_host_async")
        self._inflight.append(keep)
        return out[: g.edges]

    def wait(self):
        """Wait for every run_host_async call since the last wait."""
        try:
            _check(self._lib.ecl_mst_ctx_wait(self.handle), "ctx_wait")
        finally:
            self._inflight = []

    def run_device(self, nodes, edges, d_nindex, d_nlist, d_eweight, d_inMST, opts=None, stream=None,
                   stats=False):
        """Device pointers in and out (ints). Enqueues; returns stats only if asked."""
        gs = EclGraphC(nodes, edges, d_nindex, d_nlist, d_eweight)
        st = MstStats() if stats else None
        _check(self._lib.ecl_mst_run_device(self.handle, ctypes.byref(gs), d_inMST,
                                            None if opts is None else ctypes.byref(opts), stream,
                                            None if st is None else ctypes.byref(st)), "run_device")
        return st.as_dict() if st is not None else None

    def sync(self):
        _check(self._lib.ecl_mst_ctx_sync(self.handle), "ctx_sync")

    def l2_reset(self):
        """Return L2 lines marked persisting (FLAG_L2_PERSIST) to normal."""
        _check(self._lib.ecl_mst_ctx_l2_reset(self.handle), "ctx_l2_reset")

    def learned_features(self):
        """The 16 features the last learned-schedule solve fed its network."""
        out = np.zeros(MLP_IN, np.float32)
        _check(self._lib.ecl_mst_ctx_learned_features(self.handle, _ptr(out)), "ctx_learned_features")
        return out


class Batch:
    """Host-side packing of many graphs into one batch layout (ecl_batch).

    Segments start at multiples of `align` entries so 128-bit loads stay
    aligned; nindex of graph g sits at nindex_off[g], its entries at edge_off[g].
    """

    def __init__(self, graphs, align=4):
        self.num_graphs = len(graphs)
        self.nodes = np.array([g.nodes for g in graphs], np.int32)
        self.edges = np.array([g.edges for g in graphs], np.int32)
        noff, eoff = [], []
        no = eo = 0
        for g in graphs:
            noff.append(no)
            eoff.append(eo)
            no += -(-(g.nodes + 1) // align) * align
            eo += -(-max(g.edges, 1) // align) * align
        self.nindex_off = np.array(noff, np.int64)
        self.edge_off = np.array(eoff, np.int64)
        self.total_nindex, self.total_edges = no, eo
        self.nindex = np.zeros(no, np.int32)
        self.nlist = np.zeros(eo, np.int32)
        self.eweight = np.zeros(eo, np.int32)
        for g, a, b in zip(graphs, noff, eoff):
            self.nindex[a:a + g.nodes + 1] = g.nindex
            self.nlist[b:b + g.edges] = g.nlist
            self.eweight[b:b + g.edges] = g.eweight

    def struct(self, d_nindex, d_nlist, d_eweight):
        return EclBatchC(self.num_graphs, _ptr(self.nodes), _ptr(self.edges), _ptr(self.nindex_off),
                         _ptr(self.edge_off), d_nindex, d_nlist, d_eweight)

    def slice(self, inmst, g):
        a = int(self.edge_off[g])
        return inmst[a:a + int(self.edges[g])]

    def select(self, idx):
        """A view of graphs `idx` of this batch (see ``BatchView``)."""
        return BatchView(self, idx)


class BatchView:
    """Graphs `idx` of a packed batch (``Batch`` or ``DeviceBatch``), in that
    order, without copying their entries: the per-graph tables are subsets of
    the parent's, so the view's graphs read the parent's packed arrays and
    write their inMST at the parent's offsets of a full-size output buffer
    (``total_edges`` is the parent's). This is how a rank solves its shard of
    a batch (shard.partition_by_cost)."""

    def __init__(self, parent, idx):
        self.parent = parent
        self.idx = np.asarray(idx, np.int64)
        self.num_graphs = len(self.idx)
        self.nodes = np.ascontiguousarray(parent.nodes[self.idx], np.int32)
        self.edges = np.ascontiguousarray(parent.edges[self.idx], np.int32)
        self.nindex_off = np.ascontiguousarray(parent.nindex_off[self.idx], np.int64)
        self.edge_off = np.ascontiguousarray(parent.edge_off[self.idx], np.int64)
        self.total_nindex, self.total_edges = parent.total_nindex, parent.total_edges

    def struct(self, d_nindex=None, d_nlist=None, d_eweight=None):
        """The view as an ecl_batch; device pointers default to a DeviceBatch parent's."""
        d_nindex = d_nindex or getattr(self.parent, "d_nindex", None)
        d_nlist = d_nlist or getattr(self.parent, "d_nlist", None)
        d_eweight = d_eweight or getattr(self.parent, "d_eweight", None)
        return EclBatchC(self.num_graphs, _ptr(self.nodes), _ptr(self.edges), _ptr(self.nindex_off),
                         _ptr(self.edge_off), d_nindex, d_nlist, d_eweight)

    def slice(self, inmst, k):
        """Graph k of the view's inMST entries in a full-size output buffer."""
        return self.parent.slice(inmst, int(self.idx[k]))


class BatchContext:
    """Workspace of the batched engine (ecl_batch_ctx)."""

    def __init__(self, max_graphs, max_graph_nodes, max_graph_edges, small_cap=0, device=0):
        self._lib = load()
        h = c_void_p()
        _check(self._lib.ecl_batch_ctx_create(device, max_graphs, max_graph_nodes, max_graph_edges, small_cap,
                                              ctypes.byref(h)), "batch_ctx_create")
        self.handle = h

    def close(self):
        if self.handle:
            self._lib.ecl_batch_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def run(self, batch, d_nindex, d_nlist, d_eweight, d_inMST, opts=None, stream=None):
        bs = batch.struct(d_nindex, d_nlist, d_eweight)
        st = BatchStats()
        _check(self._lib.ecl_mst_run_batch_device(self.handle, ctypes.byref(bs), d_inMST,
                                                  None if opts is None else ctypes.byref(opts), stream,
                                                  ctypes.byref(st)), "run_batch")
        return st.as_dict()

    def autotune(self, batch, d_nindex, d_nlist, d_eweight, d_inMST, base=None):
        bs = batch.struct(d_nindex, d_nlist, d_eweight)
        best = MstOpts()
        ms = c_float()
        _check(self._lib.ecl_batch_autotune(self.handle, ctypes.byref(bs), d_inMST,
                                            None if base is None else ctypes.byref(base), ctypes.byref(best),
                                            ctypes.byref(ms)), "batch_autotune")
        return best, ms.value


# ----------------------------------------------------------- learned schedule
MLP_IN, MLP_H, MLP_OUT = 16, 64, 2
MLP_PARAMS = MLP_IN * MLP_H + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H * MLP_OUT + MLP_OUT + 2 * MLP_IN
MLP_TRAINABLE = MLP_PARAMS - 2 * MLP_IN
WEIGHTS_PATH = os.path.join(_HERE, "filter_weights.bin")


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def mlp_init(seed=0, mean=None, std=None):
    """He-initialised parameter blob (W1, b1, W2, b2, W3, b3, mean, std)."""
    rng = np.random.default_rng(seed)
    parts = [rng.normal(0, np.sqrt(2 / MLP_IN), MLP_IN * MLP_H), np.zeros(MLP_H),
             rng.normal(0, np.sqrt(2 / MLP_H), MLP_H * MLP_H), np.zeros(MLP_H),
             rng.normal(0, np.sqrt(1 / MLP_H), MLP_H * MLP_OUT), np.zeros(MLP_OUT),
             np.zeros(MLP_IN) if mean is None else mean, np.ones(MLP_IN) if std is None else std]
    return _f32(np.concatenate(parts))


def mlp_forward(params, x):
    """CUDA inference: raw features (B x 16) -> outputs (B x 2)."""
    params, x = _f32(params), _f32(x)
    y = np.zeros((x.shape[0], MLP_OUT), np.float32)
    _check(load().ecl_mlp_forward(_ptr(params), _ptr(x), x.shape[0], _ptr(y)), "mlp_forward")
    return y


def mlp_grad(params, x, t):
    """CUDA full-batch MSE gradient of W1..b3 (standardised inputs)."""
    params, x, t = _f32(params), _f32(x), _f32(t)
    g = np.zeros(MLP_TRAINABLE, np.float32)
    loss = c_float()
    _check(load().ecl_mlp_grad(_ptr(params), _ptr(x), _ptr(t), x.shape[0], _ptr(g), ctypes.byref(loss)),
           "mlp_grad")
    return g, loss.value


def mlp_train(params, x, t, epochs, lr):
    """CUDA Adam training run (standardised inputs); returns (params, loss per epoch)."""
    params = _f32(params).copy()
    x, t = _f32(x), _f32(t)
    hist = np.zeros(epochs, np.float32)
    _check(load().ecl_mlp_train(_ptr(params), _ptr(x), _ptr(t), x.shape[0], epochs, lr, _ptr(hist)),
           "mlp_train")
    return params, hist


def graph_features(nodes, edges, d_nindex, d_nlist, d_eweight):
    """The 16 schedule features of a device-resident graph (computed on the GPU)."""
    out = np.zeros(MLP_IN, np.float32)
    gs = EclGraphC(nodes, edges, d_nindex, d_nlist, d_eweight)
    _check(load().ecl_graph_features(ctypes.byref(gs), _ptr(out)), "graph_features")
    return out


def learned_set_weights(params):
    params = _f32(params)
    _check(load().ecl_learned_set_weights(_ptr(params), params.size), "learned_set_weights")


def learned_load_default():
    """Load the trained weights shipped next to this module; False if absent."""
    if not os.path.exists(WEIGHTS_PATH):
        return False
    learned_set_weights(np.fromfile(WEIGHTS_PATH, np.float32))
    return True
