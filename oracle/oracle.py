"""ctypes wrapper over oracle/liboracle.so -- the CPU parity checker.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / --impl reference legs of bench.py.  The product never imports it.
The C restatement it wraps cites the reference file:line for every step
(oracle/vann_oracle.c).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

BLOOM_CHUNK32, BLOOM_SEQUENTIAL, BLOOM_SNAPSHOT = 0, 1, 2
NONE = 0xFFFFFFFF


class _Graph(C.Structure):
    _fields_ = [
        ("vecs", C.c_void_p),
        ("n", C.c_int64),
        ("dim", C.c_int32),
        ("deg", C.c_void_p),
        ("adj", C.c_void_p),
        ("R", C.c_int32),
        ("tomb", C.c_void_p),
    ]


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.vo_bf_h1.restype = C.c_uint32
        L.vo_bf_h1.argtypes = [C.c_uint32]
        L.vo_bf_h2.restype = C.c_uint32
        L.vo_bf_h2.argtypes = [C.c_uint32]
        L.vo_medoid.restype = C.c_int64
        L.vo_medoid.argtypes = [C.c_void_p, C.c_int64, C.c_int]
        L.vo_search_batch.restype = C.c_int
        L.vo_search_batch.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                      C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.vo_search_one.restype = C.c_int
        L.vo_search_one.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_int, C.c_uint32, C.c_uint32,
                                    C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        L.vo_robust_prune.restype = C.c_int
        L.vo_robust_prune.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                      C.c_float, C.c_int, C.c_void_p, C.c_void_p]
        L.vo_vamana_batch.restype = C.c_int
        L.vo_vamana_batch.argtypes = [C.POINTER(_Graph), C.c_int64, C.c_int64, C.c_int, C.c_float,
                                      C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.vo_vamana_batch_ids.restype = C.c_int
        L.vo_vamana_batch_ids.argtypes = [C.POINTER(_Graph), C.c_void_p, C.c_int64, C.c_int, C.c_float,
                                          C.c_uint32, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.vo_consolidate.restype = C.c_int
        L.vo_consolidate.argtypes = [C.POINTER(_Graph), C.c_float, C.c_int, C.c_void_p, C.c_uint32,
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.vo_random_graph.restype = None
        L.vo_random_graph.argtypes = [C.c_int64, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p]
        L.vo_bruteforce_knn.restype = None
        L.vo_bruteforce_knn.argtypes = [C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_int]
        L.vo_u8_grid.restype = C.c_int
        L.vo_u8_grid.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.POINTER(C.c_float),
                                 C.POINTER(C.c_float)]
        L.vo_u8_codes.restype = None
        L.vo_u8_codes.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p, C.c_float, C.c_void_p]
        L.vo_merge_rerank.restype = None
        L.vo_merge_rerank.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int64, C.c_void_p, C.c_int,
                                      C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Graph:
    """Host copy of an index: vectors, degrees, adjacency (n x R), tombstones."""

    def __init__(self, vecs: np.ndarray, deg: np.ndarray, adj: np.ndarray, tomb: np.ndarray | None = None):
        self.vecs = np.ascontiguousarray(vecs, dtype=np.float32)
        self.deg = np.ascontiguousarray(deg, dtype=np.uint32)
        self.adj = np.ascontiguousarray(adj, dtype=np.uint32)
        self.tomb = None if tomb is None else np.ascontiguousarray(tomb, dtype=np.uint32)

    @property
    def n(self):
        return self.vecs.shape[0]

    @property
    def R(self):
        return self.adj.shape[1]

    def _c(self):
        return _Graph(_p(self.vecs), self.n, self.vecs.shape[1], _p(self.deg), _p(self.adj), self.R,
                      _p(self.tomb))

    def search(self, q, L, k, entry, skip_mode=0, bloom_mode=BLOOM_CHUNK32, max_hops=1 << 30, threads=0,
               with_adjw=False):
        """-> status, ids, dists, hops, evals (and with_adjw the adjacency words read)."""
        q = np.ascontiguousarray(q, dtype=np.float32)
        nq = q.shape[0]
        ids = np.empty((nq, k), np.uint32)
        d = np.empty((nq, k), np.float32)
        hops = np.empty(nq, np.int32)
        evals = np.empty(nq, np.int64)
        adjw = np.empty(nq, np.int64)
        g = self._c()
        st = lib().vo_search_batch(C.byref(g), _p(q), nq, L, k, entry, skip_mode, bloom_mode, max_hops,
                                   _p(ids), _p(d), _p(hops), _p(evals), _p(adjw), threads)
        return (st, ids, d, hops, evals, adjw) if with_adjw else (st, ids, d, hops, evals)

    def search_one(self, q, L, entry, skip_id=NONE, bloom_mode=BLOOM_CHUNK32, max_visited=600,
                   max_hops=1 << 30):
        q = np.ascontiguousarray(q, dtype=np.float32)
        wi = np.empty(L, np.uint32)
        wd = np.empty(L, np.float32)
        wn = C.c_int(0)
        vi = np.empty(max_visited, np.uint32)
        vd = np.empty(max_visited, np.float32)
        vn = C.c_int(0)
        hops = C.c_int(0)
        ev = C.c_int64(0)
        g = self._c()
        st = lib().vo_search_one(C.byref(g), _p(q), L, entry, skip_id, bloom_mode, max_visited, max_hops,
                                 _p(wi), _p(wd), C.byref(wn), _p(vi), _p(vd), C.byref(vn), C.byref(hops),
                                 C.byref(ev), None)
        return st, wi[: wn.value], wd[: wn.value], vi[: vn.value], vd[: vn.value], hops.value, ev.value

    def robust_prune(self, node_vec, cand, cand_d, alpha, R):
        cand = np.ascontiguousarray(cand, dtype=np.uint32)
        cand_d = np.ascontiguousarray(cand_d, dtype=np.float32)
        out = np.empty(R, np.uint32)
        g = self._c()
        nv = np.ascontiguousarray(node_vec, dtype=np.float32)
        d = lib().vo_robust_prune(C.byref(g), _p(nv), _p(cand), _p(cand_d), len(cand), alpha, R, _p(out), None)
        return out[:d]

    def consolidate(self, alpha, cap, entry, is_free=None, threads=0):
        """FreshVamana delete consolidation of the ids marked in self.tomb (vo_consolidate):
        updates deg/adj in place; -> (new entry, ids freed by this call, ascending)."""
        assert self.tomb is not None
        g = self._c()
        free_mask = None if is_free is None else np.ascontiguousarray(is_free, dtype=np.uint8)
        freed = np.empty(max(self.n, 1), np.uint32)
        nf = C.c_int64(0)
        ne = C.c_uint32(0)
        st = lib().vo_consolidate(C.byref(g), alpha, cap, _p(free_mask), entry, C.byref(ne), _p(freed),
                                  C.byref(nf), threads)
        assert st == 0, st
        return int(ne.value), freed[: nf.value].copy()

    def vamana_batch_ids(self, ids, L, alpha, entry, max_visited=600, max_reverse=500, skip_mode=0,
                         bloom_mode=BLOOM_SNAPSHOT, threads=0):
        """One Vamana batch over the node ids `ids` in that order (their rows already in
        self.vecs, their degrees 0): inserts into reused ids."""
        nodes = np.ascontiguousarray(ids, dtype=np.uint32)
        g = self._c()
        return lib().vo_vamana_batch_ids(C.byref(g), _p(nodes), len(nodes), L, alpha, entry, max_visited,
                                         max_reverse, skip_mode, bloom_mode, threads)

    def vamana_batch(self, batch_start, batch_n, L, alpha, entry, max_visited=600, max_reverse=500,
                     skip_mode=1, bloom_mode=BLOOM_CHUNK32, threads=0):
        g = self._c()
        return lib().vo_vamana_batch(C.byref(g), batch_start, batch_n, L, alpha, entry, max_visited,
                                     max_reverse, skip_mode, bloom_mode, threads)


def tomb_bitmap(n: int, ids) -> np.ndarray:
    """Tombstone bitmap of n ids (bit i of word i >> 5) with `ids` set."""
    t = np.zeros((n + 31) // 32, np.uint32)
    for i in np.asarray(ids, dtype=np.int64).tolist():
        t[i >> 5] |= np.uint32(1 << (i & 31))
    return t


def bf_h1(x: int) -> int:
    return lib().vo_bf_h1(x)


def bf_h2(x: int) -> int:
    return lib().vo_bf_h2(x)


def random_graph(n: int, R: int, seed: int):
    deg = np.empty(n, np.uint32)
    adj = np.empty((n, R), np.uint32)
    lib().vo_random_graph(n, R, seed, _p(deg), _p(adj))
    return deg, adj


def medoid(vecs: np.ndarray) -> int:
    v = np.ascontiguousarray(vecs, dtype=np.float32)
    return int(lib().vo_medoid(_p(v), v.shape[0], v.shape[1]))


def bruteforce_knn(base: np.ndarray, q: np.ndarray, k: int, threads: int = 0):
    base = np.ascontiguousarray(base, dtype=np.float32)
    q = np.ascontiguousarray(q, dtype=np.float32)
    ids = np.empty((q.shape[0], k), np.uint32)
    d = np.empty((q.shape[0], k), np.float64)
    lib().vo_bruteforce_knn(_p(base), base.shape[0], _p(q), q.shape[0], base.shape[1], k, _p(ids), _p(d), threads)
    return ids, d


STAGED = 0x80000000


def merge_rerank(vecs: np.ndarray, q: np.ndarray, graph_ids: np.ndarray, insert_list: np.ndarray):
    """searchPoints2's merge of the L graph results with the insert list
    (utils.cuh:199-285): ids (insert-list row s as STAGED | s) and distances, n x L."""
    vecs = np.ascontiguousarray(vecs, dtype=np.float32)
    q = np.ascontiguousarray(q, dtype=np.float32)
    gi = np.ascontiguousarray(graph_ids, dtype=np.uint32)
    il = np.ascontiguousarray(insert_list, dtype=np.float32).reshape(-1, vecs.shape[1])
    nq, L = gi.shape
    ids = np.empty((nq, L), np.uint32)
    d = np.empty((nq, L), np.float32)
    lib().vo_merge_rerank(_p(vecs), vecs.shape[1], _p(q), nq, _p(gi), L, _p(il) if len(il) else None,
                          len(il), _p(ids), _p(d))
    return ids, d


def build_index(vecs, R, L, alpha, entry=None, seed=0, skip_mode=1, bloom_mode=BLOOM_CHUNK32,
                max_visited=600, max_reverse=500, threads=0):
    """Reference build (vamana_impl.cuh:289-360 runVamana): one batch of all nodes
    over a seeded random R-regular start graph."""
    n = vecs.shape[0]
    deg, adj = random_graph(n, R, seed)
    g = Graph(vecs, deg, adj)
    if entry is None:
        entry = medoid(vecs)
    st = g.vamana_batch(0, n, L, alpha, entry, max_visited, max_reverse, skip_mode, bloom_mode, threads)
    assert st == 0, st
    return g, entry


def recall_at_k(found: np.ndarray, truth: np.ndarray, k: int) -> float:
    hit = 0
    for f, t in zip(found[:, :k], truth[:, :k]):
        hit += len(set(f.tolist()) & set(t.tolist()))
    return hit / (truth.shape[0] * k)


def u8_grid(vecs: np.ndarray):
    """The uint8 copy's grid fitted to `vecs` (vo_u8_grid): (fitted, lo[dim], s, inv);
    fitted False means the identity grid (every value an integer in [0, 255])."""
    v = np.ascontiguousarray(vecs, dtype=np.float32)
    lo = np.empty(v.shape[1], np.float32)
    s, inv = C.c_float(), C.c_float()
    fitted = lib().vo_u8_grid(_p(v), v.shape[0], v.shape[1], _p(lo), C.byref(s), C.byref(inv))
    return bool(fitted), lo, np.float32(s.value), np.float32(inv.value)


def u8_codes(x: np.ndarray, lo, inv) -> np.ndarray:
    """Codes of rows or queries on a grid (vo_u8_codes); lo None: the identity grid."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    out = np.empty(x.shape, np.uint8)
    lo_c = None if lo is None else np.ascontiguousarray(lo, dtype=np.float32)
    lib().vo_u8_codes(_p(x), x.shape[0], x.shape[1], _p(lo_c), float(inv), _p(out))
    return out
