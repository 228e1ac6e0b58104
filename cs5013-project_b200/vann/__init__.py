"""Python host mirror of the B200-native Vamana / FreshVamana engine.

Thin ctypes layer over libvann.so (the C ABI in include/vann.h).  Device
memory and streams come from torch; every computation runs in the library's
CUDA kernels.  There is no CPU fallback: importing this module on a machine
without the built library raises.

Two layers:
  * ``Index``   -- one vann_index handle, pythonic names.
  * ``Vamana``  -- the reference's class interface (vamana/include/vamana.cuh:36-146):
                   searchPoints / insertPoints / deletePoints / patchGraph /
                   saveGraph, with the reference's staging semantics for inserts.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvann.so")

OK, ERR_INVALID, ERR_CUDA, ERR_CAPACITY, ERR_IO, ERR_HOP_LIMIT = 0, 1, 2, 3, 4, 5
ERR_NOT_FOUND, ERR_TIMEOUT, ERR_OOM, ERR_UNSUPPORTED, ERR_STATE = 6, 7, 8, 9, 10
STORE_F32, STORE_BF16, STORE_FP8, STORE_U8, STORE_PQ = 0, 1, 2, 3, 4
STORES = {"f32": STORE_F32, "bf16": STORE_BF16, "fp8": STORE_FP8, "u8": STORE_U8, "pq": STORE_PQ}
QUIRK_SKIP_BATCH_INDEX = 0x1
NONE_ID = 0xFFFFFFFF
STAGED_BIT = 0x80000000  # VANN_STAGED_ID(s): insert-list row s in vann_search_staged results

# every symbol include/vann.h declares
EXPORTS = [
    "vann_status_string", "vann_last_error", "vann_abi_version", "vann_create", "vann_destroy",
    "vann_get_info", "vann_load_graph", "vann_save_graph", "vann_set_graph", "vann_get_graph",
    "vann_build", "vann_build_loaded", "vann_search", "vann_search_stats", "vann_search_uneven", "vann_autotune", "vann_search_variant_count", "vann_sync", "vann_insert", "vann_delete", "vann_delete_by_vector",
    "vann_consolidate", "vann_medoid_noalloc", "vann_server_create", "vann_server_destroy",
    "vann_server_submit_search", "vann_server_submit_insert", "vann_server_submit_delete",
    "vann_server_submit_consolidate", "vann_server_wait", "vann_server_get_stats",
    "vann_stage_insert", "vann_search_staged", "vann_patch_graph", "vann_convert_graph_file",
    "vann_save_graph_bang", "vann_save_index", "vann_load_index",
]


class VannError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"vann status {status}: {msg}")
        self.status = status


class Params(C.Structure):
    _fields_ = [("dim", C.c_uint32), ("degree", C.c_uint32), ("build_L", C.c_uint32),
                ("alpha", C.c_float), ("capacity", C.c_uint64), ("max_visited", C.c_uint32),
                ("max_reverse", C.c_uint32), ("flags", C.c_uint32), ("stores", C.c_uint32)]


class SearchParams(C.Structure):
    _fields_ = [("L", C.c_uint32), ("k", C.c_uint32), ("store", C.c_uint32), ("rerank", C.c_uint32),
                ("flags", C.c_uint32), ("max_hops", C.c_uint32), ("beam", C.c_uint32)]


class Info(C.Structure):
    _fields_ = [("size", C.c_uint64), ("capacity", C.c_uint64), ("live", C.c_uint64),
                ("free_ids", C.c_uint64), ("entry", C.c_uint32), ("dim", C.c_uint32),
                ("degree", C.c_uint32), ("consistent", C.c_uint32), ("device_bytes", C.c_uint64),
                ("pruned_tc", C.c_uint64), ("pruned_cuda", C.c_uint64), ("staged", C.c_uint64)]


class ServerParams(C.Structure):
    _fields_ = [("max_batch", C.c_uint32), ("slots", C.c_uint32), ("hbm_budget", C.c_uint64),
                ("max_k", C.c_uint32), ("store", C.c_uint32), ("rerank", C.c_uint32),
                ("commit_interval_us", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [("slots", C.c_uint32), ("slot_bytes", C.c_uint64), ("batches", C.c_uint64),
                ("queries", C.c_uint64), ("writes", C.c_uint64), ("max_inflight", C.c_uint64),
                ("queued", C.c_uint64), ("epoch", C.c_uint64)]


_lib = None
ABI_VERSION = 2  # VANN_ABI_VERSION of include/vann.h that these ctypes structs mirror


def lib():
    """Load libvann.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run cs5013-project_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp, u64, u32 = C.c_void_p, C.c_uint64, C.c_uint32
        sig = {
            "vann_status_string": (C.c_char_p, [C.c_int]),
            "vann_last_error": (C.c_char_p, []),
            "vann_abi_version": (C.c_int, []),
            "vann_create": (C.c_int, [C.POINTER(Params), C.POINTER(vp)]),
            "vann_destroy": (C.c_int, [vp]),
            "vann_get_info": (C.c_int, [vp, C.POINTER(Info)]),
            "vann_load_graph": (C.c_int, [vp, C.c_char_p, u64, u32]),
            "vann_save_graph": (C.c_int, [vp, C.c_char_p]),
            "vann_set_graph": (C.c_int, [vp, vp, vp, vp, u64, u32, u32]),
            "vann_get_graph": (C.c_int, [vp, vp, vp, vp]),
            "vann_build": (C.c_int, [vp, vp, u64, u64, u64, u32, vp]),
            "vann_build_loaded": (C.c_int, [vp, vp]),
            "vann_search": (C.c_int, [vp, vp, u64, C.POINTER(SearchParams), vp, vp, vp]),
            "vann_search_stats": (C.c_int, [vp, vp, u64, C.POINTER(SearchParams), vp, vp, vp, vp, vp, vp]),
            "vann_search_uneven": (C.c_int, [vp, vp, u64, C.POINTER(SearchParams), vp, vp, vp, vp, vp]),
            "vann_autotune": (C.c_int, [vp, vp, u64, C.POINTER(SearchParams), vp, vp]),
            "vann_search_variant_count": (C.c_int, []),
            "vann_sync": (C.c_int, [vp, vp]),
            "vann_insert": (C.c_int, [vp, vp, u64, vp, vp]),
            "vann_delete": (C.c_int, [vp, vp, u64, vp]),
            "vann_delete_by_vector": (C.c_int, [vp, vp, u64, vp, vp]),
            "vann_consolidate": (C.c_int, [vp, vp]),
            "vann_medoid_noalloc": (C.c_int, [vp, u64, u32, vp, vp]),
            "vann_server_create": (C.c_int, [vp, C.POINTER(ServerParams), C.POINTER(vp)]),
            "vann_server_destroy": (C.c_int, [vp]),
            "vann_server_submit_search": (C.c_int, [vp, vp, u32, u32, u32, C.POINTER(u64)]),
            "vann_server_submit_insert": (C.c_int, [vp, vp, u32, C.POINTER(u64)]),
            "vann_server_submit_delete": (C.c_int, [vp, vp, u32, C.POINTER(u64)]),
            "vann_server_submit_consolidate": (C.c_int, [vp, C.POINTER(u64)]),
            "vann_server_wait": (C.c_int, [vp, u64, vp, vp, C.POINTER(C.c_double), C.POINTER(u64), u32]),
            "vann_server_get_stats": (C.c_int, [vp, C.POINTER(ServerStats)]),
            "vann_stage_insert": (C.c_int, [vp, vp, u64, vp]),
            "vann_search_staged": (C.c_int, [vp, vp, u64, C.POINTER(SearchParams), vp, vp, vp, vp]),
            "vann_patch_graph": (C.c_int, [vp, vp, vp]),
            "vann_convert_graph_file": (C.c_int, [C.c_char_p, u64, u32, u32, u32, C.c_char_p]),
            "vann_save_graph_bang": (C.c_int, [vp, C.c_char_p]),
            "vann_save_index": (C.c_int, [vp, C.c_char_p]),
            "vann_load_index": (C.c_int, [vp, C.c_char_p]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        if L.vann_abi_version() != ABI_VERSION:  # the structs below must match the library's
            raise ImportError(f"{LIB_PATH} has C ABI {L.vann_abi_version()}, this module needs {ABI_VERSION}")
        _lib = L
    return _lib


def _check(st: int):
    if st != OK:
        raise VannError(st, lib().vann_last_error().decode())


def _torch():
    import torch
    return torch


def _stream_ptr(stream):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev(t, dtype):
    torch = _torch()
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise TypeError(f"expected a contiguous CUDA tensor of {dtype}")
    return C.c_void_p(t.data_ptr())


class Index:
    """One device-resident Vamana index (vann_index)."""

    def __init__(self, dim: int, degree: int = 64, build_L: int = 100, alpha: float = 1.2,
                 capacity: int = 1 << 20, max_visited: int = 600, max_reverse: int = 500,
                 quirks: int = 0, stores=("f32",)):
        mask = 0
        for s in stores:
            if s != "f32":
                mask |= 1 << STORES[s]
        p = Params(dim, degree, build_L, alpha, capacity, max_visited, max_reverse, quirks, mask)
        h = C.c_void_p()
        _check(lib().vann_create(C.byref(p), C.byref(h)))
        self._h = h
        self.dim, self.degree = dim, degree

    def close(self):
        if getattr(self, "_h", None):
            lib().vann_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- graph I/O
    def info(self) -> dict:
        i = Info()
        _check(lib().vann_get_info(self._h, C.byref(i)))
        return {f: getattr(i, f) for f, _ in Info._fields_}

    def set_graph(self, vecs, deg, adj, entry: int, consistent: bool = False):
        import numpy as np
        vecs = np.ascontiguousarray(vecs, dtype=np.float32)
        deg = np.ascontiguousarray(deg, dtype=np.uint32)
        adj = np.ascontiguousarray(adj, dtype=np.uint32)
        assert adj.shape[1] == self.degree and vecs.shape[1] == self.dim
        _check(lib().vann_set_graph(self._h, vecs.ctypes.data, deg.ctypes.data, adj.ctypes.data,
                                    vecs.shape[0], entry, int(consistent)))

    def get_graph(self):
        import numpy as np
        n = self.info()["size"]
        vecs = np.empty((n, self.dim), np.float32)
        deg = np.empty(n, np.uint32)
        adj = np.empty((n, self.degree), np.uint32)
        _check(lib().vann_get_graph(self._h, vecs.ctypes.data, deg.ctypes.data, adj.ctypes.data))
        return vecs, deg, adj

    def load_graph(self, path: str, n: int, entry: int):
        _check(lib().vann_load_graph(self._h, path.encode(), n, entry))

    def save_graph(self, path: str):
        _check(lib().vann_save_graph(self._h, path.encode()))

    # ---------------------------------------------------------------- hot path
    def build(self, vecs, batch: int = 0, seed: int = 0, entry: int | None = None, stream=None):
        torch = _torch()
        _check(lib().vann_build(self._h, _dev(vecs, torch.float32), vecs.shape[0], batch, seed,
                                NONE_ID if entry is None else entry, _stream_ptr(stream)))

    def build_loaded(self, stream=None):
        """Reference build over the graph already loaded (its adjacency is the start graph)."""
        _check(lib().vann_build_loaded(self._h, _stream_ptr(stream)))

    def search(self, queries, k: int, L: int, store: str = "f32", rerank: bool = False,
               quirks: int = 0, max_hops: int = 0, out=None, stream=None, beam: int = 1):
        """Batched search; beam=2 expands two parents per hop (a batched form with its
        own results; beam=1 is the reference's GreedySearch)."""
        torch = _torch()
        nq = queries.shape[0]
        if out is None:
            ids = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
            dists = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
        else:
            ids, dists = out
        sp = SearchParams(L, k, STORES[store], int(rerank), quirks, max_hops, beam)
        _check(lib().vann_search(self._h, _dev(queries, torch.float32), nq, C.byref(sp),
                                 _dev(ids, torch.int32), _dev(dists, torch.float32), _stream_ptr(stream)))
        return ids, dists

    def search_uneven(self, queries, L, k, store: str = "f32", rerank: bool = False, quirks: int = 0,
                      stream=None, beam: int = 1):
        """One launch over queries with their own L[i] and k[i] (int32 CUDA tensors);
        returns (ids, dists) with max(k) columns, padded past k[i]."""
        torch = _torch()
        nq = queries.shape[0]
        Lmax, kmax = int(L.max().item()), int(k.max().item())
        ids = torch.empty((nq, kmax), dtype=torch.int32, device=queries.device)
        dists = torch.empty((nq, kmax), dtype=torch.float32, device=queries.device)
        sp = SearchParams(Lmax, kmax, STORES[store], int(rerank), quirks, 0, beam)
        _check(lib().vann_search_uneven(self._h, _dev(queries, torch.float32), nq, C.byref(sp),
                                        _dev(L, torch.int32), _dev(k, torch.int32), _dev(ids, torch.int32),
                                        _dev(dists, torch.float32), _stream_ptr(stream)))
        return ids, dists

    def search_stats(self, queries, k: int, L: int, store: str = "f32", rerank: bool = False,
                     quirks: int = 0, max_hops: int = 0, stream=None, beam: int = 1):
        """search() plus per-query (hops, distance evaluations, adjacency words)."""
        torch = _torch()
        nq = queries.shape[0]
        ids = torch.empty((nq, k), dtype=torch.int32, device=queries.device)
        dists = torch.empty((nq, k), dtype=torch.float32, device=queries.device)
        st = torch.empty((3, nq), dtype=torch.int32, device=queries.device)
        sp = SearchParams(L, k, STORES[store], int(rerank), quirks, max_hops, beam)
        _check(lib().vann_search_stats(self._h, _dev(queries, torch.float32), nq, C.byref(sp),
                                       _dev(ids, torch.int32), _dev(dists, torch.float32),
                                       C.c_void_p(st[0].data_ptr()), C.c_void_p(st[1].data_ptr()),
                                       C.c_void_p(st[2].data_ptr()), _stream_ptr(stream)))
        return ids, dists, st

    def autotune(self, queries, k: int, L: int, store: str = "f32", rerank: bool = False, quirks: int = 0,
                 stream=None, beam: int = 1):
        """Pick the fastest compiled search variant for (store, rerank, beam, L) on these queries."""
        torch = _torch()
        sp = SearchParams(L, k, STORES[store], int(rerank), quirks, 0, beam)
        nv = lib().vann_search_variant_count()
        ms = (C.c_float * nv)()
        _check(lib().vann_autotune(self._h, _dev(queries, torch.float32), queries.shape[0], C.byref(sp),
                                   ms, _stream_ptr(stream)))
        return [round(float(x), 4) for x in ms]

    def sync(self, stream=None):
        _check(lib().vann_sync(self._h, _stream_ptr(stream)))

    def insert(self, vecs, stream=None):
        torch = _torch()
        ids = torch.empty(vecs.shape[0], dtype=torch.int32, device=vecs.device)
        _check(lib().vann_insert(self._h, _dev(vecs, torch.float32), vecs.shape[0], _dev(ids, torch.int32),
                                 _stream_ptr(stream)))
        return ids

    def delete(self, ids, stream=None):
        torch = _torch()
        _check(lib().vann_delete(self._h, _dev(ids, torch.int32), ids.shape[0], _stream_ptr(stream)))

    def delete_by_vector(self, vecs, stream=None):
        torch = _torch()
        out = torch.empty(vecs.shape[0], dtype=torch.int32, device=vecs.device)
        st = lib().vann_delete_by_vector(self._h, _dev(vecs, torch.float32), vecs.shape[0],
                                         _dev(out, torch.int32), _stream_ptr(stream))
        if st not in (OK, ERR_NOT_FOUND):
            _check(st)
        return out

    def consolidate(self, stream=None):
        _check(lib().vann_consolidate(self._h, _stream_ptr(stream)))

    def save_graph_bang(self, prefix: str):
        """<prefix>_disk.bin + <prefix>_disk_metadata.bin in the BANG / DiskANN layout."""
        _check(lib().vann_save_graph_bang(self._h, prefix.encode()))

    def save_index(self, path: str):
        """Versioned full-state file: graph, tombstones, free ids, entry, consistency."""
        _check(lib().vann_save_index(self._h, path.encode()))

    def load_index(self, path: str):
        _check(lib().vann_load_index(self._h, path.encode()))

    def stage_insert(self, vecs, stream=None):
        """Append rows to the insert list, outside the graph (vann_stage_insert)."""
        torch = _torch()
        _check(lib().vann_stage_insert(self._h, _dev(vecs, torch.float32), vecs.shape[0], _stream_ptr(stream)))

    def search_staged(self, queries, L: int, store: str = "f32", rerank: bool = False, quirks: int = 0,
                      with_vecs: bool = False, stream=None):
        """searchPoints2 (vann_search_staged): n x L graph ids or STAGED_BIT | row, distances,
        and with_vecs the n x L x dim rows."""
        torch = _torch()
        n = queries.shape[0]
        sp = SearchParams(L, L, STORES[store], int(rerank), quirks, 0)
        ids = torch.empty((n, L), dtype=torch.int32, device=queries.device)
        d = torch.empty((n, L), dtype=torch.float32, device=queries.device)
        v = torch.empty((n, L, queries.shape[1]), dtype=torch.float32, device=queries.device) if with_vecs else None
        _check(lib().vann_search_staged(self._h, _dev(queries, torch.float32), n, C.byref(sp),
                                        _dev(ids, torch.int32), _dev(d, torch.float32),
                                        _dev(v, torch.float32) if v is not None else None, _stream_ptr(stream)))
        return (ids, d, v) if with_vecs else (ids, d)

    def patch_graph(self, stream=None):
        """Move the insert list into the graph (vann_patch_graph); returns the new ids."""
        torch = _torch()
        n = self.info()["staged"]
        ids = torch.empty(n, dtype=torch.int32, device="cuda")
        _check(lib().vann_patch_graph(self._h, _dev(ids, torch.int32) if n else None, _stream_ptr(stream)))
        return ids


class Server:
    """Continuous-batching request loop over one Index (vann_server_*).  Requests
    carry host (numpy) data; submit_* return tickets, wait() returns results."""

    def __init__(self, index: "Index", max_batch: int = 4096, slots: int = 4, hbm_budget: int = 0,
                 max_k: int = 100, store: str = "f32", rerank: bool = False, commit_interval_us: int = 0):
        p = ServerParams(max_batch, slots, hbm_budget, max_k, STORES[store], int(rerank), commit_interval_us)
        h = C.c_void_p()
        _check(lib().vann_server_create(index._h, C.byref(p), C.byref(h)))
        self._h, self.index, self.dim = h, index, index.dim
        self._kind = {}

    def close(self):
        if getattr(self, "_h", None):
            lib().vann_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit_search(self, q, k: int, L: int) -> int:
        import numpy as np
        q = np.ascontiguousarray(q, dtype=np.float32).reshape(-1, self.dim)
        t = C.c_uint64()
        _check(lib().vann_server_submit_search(self._h, q.ctypes.data, q.shape[0], k, L, C.byref(t)))
        self._kind[t.value] = ("search", q.shape[0], k)
        return t.value

    def submit_insert(self, vecs) -> int:
        import numpy as np
        v = np.ascontiguousarray(vecs, dtype=np.float32).reshape(-1, self.dim)
        t = C.c_uint64()
        _check(lib().vann_server_submit_insert(self._h, v.ctypes.data, v.shape[0], C.byref(t)))
        self._kind[t.value] = ("insert", v.shape[0], 1)
        return t.value

    def submit_delete(self, ids) -> int:
        import numpy as np
        i = np.ascontiguousarray(ids, dtype=np.uint32)
        t = C.c_uint64()
        _check(lib().vann_server_submit_delete(self._h, i.ctypes.data, i.shape[0], C.byref(t)))
        self._kind[t.value] = ("delete", i.shape[0], 0)
        return t.value

    def submit_consolidate(self) -> int:
        t = C.c_uint64()
        _check(lib().vann_server_submit_consolidate(self._h, C.byref(t)))
        self._kind[t.value] = ("consolidate", 0, 0)
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 0, with_epoch: bool = False):
        """-> (ids, dists, latency_us[, epoch]); ids/dists are n x k for searches, the new
        ids for inserts; epoch = writes a search saw / a write's position in the write order."""
        import numpy as np
        kind, n, k = self._kind.pop(ticket)
        ids = np.empty((n, k), np.uint32) if kind == "search" else np.empty(n, np.uint32)
        d = np.empty((n, k), np.float32) if kind == "search" else None
        lat = C.c_double()
        ep = C.c_uint64()
        _check(lib().vann_server_wait(self._h, ticket, ids.ctypes.data if n else None,
                                      d.ctypes.data if d is not None else None, C.byref(lat), C.byref(ep),
                                      timeout_ms))
        return (ids, d, lat.value, ep.value) if with_epoch else (ids, d, lat.value)

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().vann_server_get_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in ServerStats._fields_}


def convert_graph_file(in_path: str, n: int, dim: int, degree: int, medoid: int, out_prefix: str):
    """The reference's 772-byte record file -> BANG / DiskANN disk layout, on the host
    (what scripts/bang-preprocess.py does); no GPU needed."""
    _check(lib().vann_convert_graph_file(in_path.encode(), n, dim, degree, medoid, out_prefix.encode()))


def medoid_noalloc(vecs, out, stream=None):
    """Entry point (medoid) of the rows of `vecs` written into the 1-element int32
    tensor `out`, allocating no device memory (vann_medoid_noalloc)."""
    torch = _torch()
    _check(lib().vann_medoid_noalloc(_dev(vecs, torch.float32), vecs.shape[0], vecs.shape[1],
                                     _dev(out, torch.int32), _stream_ptr(stream)))


class Vamana:
    """The reference's index class (vamana/include/vamana.cuh:36-146) on top of Index.

    ``Vamana(vecs, R, L, alpha, ...)`` builds like the reference constructor
    (vamana_impl.cuh:10-20 -> runVamana :289-360).  insertPoints appends to the
    index's insert list (vamana_impl.cuh:22-33); searchPoints2 merges graph results
    with it and returns the n x L x dim rows (:98-180); patchGraph inserts the list
    and consolidates deletes (:182-265); deletePoints matches by vector (:35-53);
    searchPoints returns the n x L worklist ids (:55-96).
    """

    def __init__(self, vecs, R: int = 64, L: int = 199, alpha: float = 1.5, capacity: int | None = None,
                 entry: int | None = None, seed: int = 0, reference_quirks: bool = True,
                 max_visited: int = 600, max_reverse: int = 500):
        self.R, self.L = R, L
        n = vecs.shape[0]
        self.quirks = QUIRK_SKIP_BATCH_INDEX if reference_quirks else 0
        self.index = Index(vecs.shape[1], R, L, alpha, capacity or max(int(n * 1.3), n + 1), max_visited,
                           max_reverse, self.quirks)
        self.index.build(vecs, batch=0, seed=seed, entry=entry)

    def insertPoints(self, d_vecs, num: int | None = None):
        self.index.stage_insert(d_vecs[: num if num is not None else d_vecs.shape[0]].contiguous())

    def deletePoints(self, d_vecs, num: int | None = None):
        return self.index.delete_by_vector(d_vecs[: num if num is not None else d_vecs.shape[0]].contiguous())

    def searchPoints(self, d_q, num: int | None = None):
        q = d_q[: num if num is not None else d_q.shape[0]].contiguous()
        ids, _ = self.index.search(q, k=self.L, L=self.L, quirks=self.quirks)
        return ids

    def searchPoints2(self, d_q, num: int | None = None):
        q = d_q[: num if num is not None else d_q.shape[0]].contiguous()
        _, _, vecs = self.index.search_staged(q, L=self.L, quirks=self.quirks, with_vecs=True)
        return vecs

    def patchGraph(self):
        self.index.patch_graph()
        self.index.consolidate()

    def saveGraph(self, path: str):
        self.index.save_graph(path)
