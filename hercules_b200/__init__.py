"""hercules_b200 -- B200-native exact k-NN for z-normalised data series.

Python binding of libhercules_gpu.so (include/hercules_gpu.h).  The index
keeps the reference Hercules EAPCA tree, leaf layout and on-disk format
(karimaechihabi/hercules, code/hercules); queries run as sm_100a kernels on
one GPU.  There is no CPU fallback: every call that computes goes through the
CUDA library and raises HerculesError when it cannot.

Names mirror the reference's C API:
  HerculesIndex.build / build_file  -> hercules_index_build (one insert worker)
  HerculesIndex.write               -> hercules_index_write_sequential
  HerculesIndex.read                -> hercules_index_read
  HerculesIndex.knn                 -> exact_de_knn_search per query
  HerculesIndex.pscan               -> the PSCAN parallel scan (code/pscan)
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libhercules_gpu.so")

MODE_PLAIN = 0
MODE_PSCAN = 1
MODE_BATCH = 2

_STATUS = {0: "ok", -1: "invalid argument", -2: "i/o error", -3: "index format error", -4: "CUDA error",
           -5: "out of memory", -6: "device wait timed out", -7: "size limit exceeded"}


class HerculesError(RuntimeError):
    def __init__(self, status, detail=""):
        self.status = status
        super().__init__("%s (%d)%s" % (_STATUS.get(status, "unknown"), status, ": " + detail if detail else ""))


class IndexInfo(ctypes.Structure):
    _fields_ = [("num_series", ctypes.c_uint64), ("ts_length", ctypes.c_uint32), ("leaf_size", ctypes.c_uint32),
                ("num_leaves", ctypes.c_uint32), ("num_nodes", ctypes.c_uint32), ("max_segments", ctypes.c_uint32),
                ("has_ids", ctypes.c_uint32), ("device_bytes", ctypes.c_uint64)]


class QueryStats(ctypes.Structure):
    _fields_ = [("queries", ctypes.c_uint64), ("leaves_scanned", ctypes.c_uint64),
                ("rows_visited", ctypes.c_uint64), ("rows_lbsax_pruned", ctypes.c_uint64),
                ("chunks_loaded", ctypes.c_uint64), ("candidate_leaves", ctypes.c_uint64),
                ("device_ms", ctypes.c_double), ("rows_completed", ctypes.c_uint64),
                ("scan_launches", ctypes.c_uint64), ("scan_ms", ctypes.c_double),
                ("rows_considered", ctypes.c_uint64), ("filter_launches", ctypes.c_uint64),
                ("filter_ms", ctypes.c_double), ("bf16_pairs", ctypes.c_uint64),
                ("survivors", ctypes.c_uint64), ("fallback_queries", ctypes.c_uint64),
                ("retried_queries", ctypes.c_uint64),
                ("bound_ms", ctypes.c_double), ("gemm_ms", ctypes.c_double), ("rerank_ms", ctypes.c_double),
                ("fallback_ms", ctypes.c_double), ("kernel_launches", ctypes.c_uint64),
                ("err_mean", ctypes.c_double), ("err_max", ctypes.c_double), ("err_over_bound", ctypes.c_double),
                ("leaf_pairs", ctypes.c_uint64), ("leaf_pairs_kept", ctypes.c_uint64)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class KnnOpts(ctypes.Structure):
    _fields_ = [("mode", ctypes.c_int), ("use_lb_sax", ctypes.c_int), ("profile", ctypes.c_int),
                ("approx_blocks", ctypes.c_int), ("bucket_cap", ctypes.c_int), ("dense_filter", ctypes.c_int),
                ("epsilon", ctypes.c_float), ("nprobes", ctypes.c_int), ("approx_leaves", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("filter_tiles_per_item", ctypes.c_uint32), ("bound_tiles_per_item", ctypes.c_uint32),
                ("rerank_blocks_per_sm", ctypes.c_uint32), ("approx_blocks_per_sm", ctypes.c_uint32),
                ("filter_cta_pair", ctypes.c_uint32), ("batch_ms", ctypes.c_double), ("plain_ms", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None

# (name, restype, argtypes) for every entry point of include/hercules_gpu.h
_P = ctypes.c_void_p
_SIGS = [
    ("hg_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("hg_last_error", ctypes.c_char_p, []),
    ("hg_index_build_file", ctypes.c_int, [ctypes.c_char_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                           ctypes.c_int, ctypes.POINTER(_P)]),
    ("hg_index_build", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_int, ctypes.POINTER(_P)]),
    ("hg_index_write", ctypes.c_int, [_P, ctypes.c_char_p, ctypes.c_double]),
    ("hg_index_read", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(_P)]),
    ("hg_index_destroy", None, [_P]),
    ("hg_index_info_get", ctypes.c_int, [_P, ctypes.POINTER(IndexInfo)]),
    ("hg_index_leaf", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    ("hg_index_leaf_envelope", ctypes.c_int, [_P, ctypes.c_uint32, _P, _P]),
    ("hg_index_row_ids", ctypes.c_int, [_P, _P]),
    ("hg_index_rows", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint64, _P, _P]),
    ("hg_knn", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(KnnOpts), _P, _P, _P,
                              ctypes.POINTER(QueryStats)]),
    ("hg_knn_device", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.POINTER(KnnOpts), _P, _P,
                                     _P, ctypes.POINTER(QueryStats)]),
    ("hg_knn_batch", ctypes.c_int, [_P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, ctypes.POINTER(KnnOpts), _P, _P,
                                    ctypes.POINTER(QueryStats)]),
    ("hg_knn_batch_device", ctypes.c_int, [_P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, ctypes.POINTER(KnnOpts),
                                           _P, _P, _P, ctypes.POINTER(QueryStats)]),
    ("hg_bf16_dots", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P]),
    ("hg_filter_wait_check", ctypes.c_int, [ctypes.c_uint32, ctypes.c_int, _P]),
    ("hg_filter_pair_wait_check", ctypes.c_int, [ctypes.c_uint32, ctypes.c_int, _P]),
    ("hg_tuning_get", ctypes.c_int, [_P, ctypes.POINTER(Tuning)]),
    ("hg_tuning_set", ctypes.c_int, [_P, ctypes.POINTER(Tuning)]),
    ("hg_autotune", ctypes.c_int, [_P, _P, ctypes.c_uint32, _P, ctypes.c_uint32, _P, ctypes.POINTER(Tuning)]),
    ("hg_route", ctypes.c_int, [_P, _P, ctypes.c_uint32, _P]),
    ("hg_leaf_lower_bounds", ctypes.c_int, [_P, _P, _P]),
    ("hg_generate_walks", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, _P,
                                         ctypes.c_int, ctypes.c_int]),
    ("hg_generate_queries", ctypes.c_int, [ctypes.c_uint64, _P, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                           _P, _P, _P, ctypes.c_int, ctypes.c_int]),
    ("hg_generate_unit_vectors", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                                _P, ctypes.c_int, ctypes.c_int]),
    ("hg_generate_unit_queries", ctypes.c_int, [ctypes.c_uint64, _P, ctypes.c_uint64, ctypes.c_uint32,
                                                ctypes.c_uint32, _P, _P, _P, ctypes.c_int, ctypes.c_int]),
    ("hg_generate_queries_seeded", ctypes.c_int, [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                                  ctypes.c_uint32, _P, ctypes.c_int, _P, _P, ctypes.c_int,
                                                  ctypes.c_int]),
    ("hg_sax_breakpoints", ctypes.c_int, [_P]),
    ("hg_pscan_noalloc", ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_uint32, _P, ctypes.c_uint32, _P, _P, _P]),
]

EXPORTED = [s[0] for s in _SIGS]


def lib():
    """The loaded libhercules_gpu.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HerculesError(-4, "libhercules_gpu.so is not built (run python hercules_b200/build.py)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _check(status):
    if status != 0:
        raise HerculesError(status, lib().hg_last_error().decode(errors="replace"))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


def _f32(a, L=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if L is not None:
        a = a.reshape(-1, L)
    return a


class HerculesIndex:
    """A resident Hercules index on one GPU."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)
        info = IndexInfo()
        _check(lib().hg_index_info_get(self._h, ctypes.byref(info)))
        self.info = info

    # -- construction ------------------------------------------------------
    @classmethod
    def build(cls, data, leaf_size, device=0):
        """hercules_index_build with one insert worker; data is n x L float32."""
        data = _f32(data)
        if data.ndim != 2:
            raise ValueError("data must be n x L")
        h = ctypes.c_void_p()
        _check(lib().hg_index_build(_ptr(data), 0, data.shape[0], data.shape[1], leaf_size, device,
                                    ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def build_device(cls, data_ptr, n, L, leaf_size, device=0):
        """Build from an n x L float32 array already resident on `device`."""
        h = ctypes.c_void_p()
        _check(lib().hg_index_build(ctypes.c_void_p(data_ptr), 1, n, L, leaf_size, device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def build_file(cls, path, n, L, leaf_size, device=0):
        h = ctypes.c_void_p()
        _check(lib().hg_index_build_file(path.encode(), n, L, leaf_size, device, ctypes.byref(h)))
        return cls(h.value)

    @classmethod
    def read(cls, directory, device=0):
        """hercules_index_read: load an index written by the reference or by write()."""
        if not directory.endswith("/"):
            directory += "/"
        h = ctypes.c_void_p()
        _check(lib().hg_index_read(directory.encode(), device, ctypes.byref(h)))
        return cls(h.value)

    def write(self, directory, buffer_mb=0.0):
        """hercules_index_write_sequential into an existing directory."""
        if not directory.endswith("/"):
            directory += "/"
        _check(lib().hg_index_write(self._h, directory.encode(), float(buffer_mb)))

    def close(self):
        if self._h:
            lib().hg_index_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- inspection ----------------------------------------------------------
    @property
    def L(self):
        return self.info.ts_length

    @property
    def n(self):
        return self.info.num_series

    def leaves(self):
        """[(file_pos, size, num_segments)] in DFS order."""
        out = []
        for i in range(self.info.num_leaves):
            fp, sz, ns = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32()
            _check(lib().hg_index_leaf(self._h, i, ctypes.byref(fp), ctypes.byref(sz), ctypes.byref(ns)))
            out.append((fp.value, sz.value, ns.value))
        return out

    def leaf_envelope(self, i):
        fp, sz, n = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().hg_index_leaf(self._h, i, ctypes.byref(fp), ctypes.byref(sz), ctypes.byref(n)))
        pts = np.zeros(n.value, dtype=np.int16)
        env = np.zeros((n.value, 4), dtype=np.float32)
        _check(lib().hg_index_leaf_envelope(self._h, i, _ptr(pts), _ptr(env)))
        return pts, env

    def row_ids(self):
        ids = np.zeros(self.n, dtype=np.int64)
        _check(lib().hg_index_row_ids(self._h, _ptr(ids)))
        return ids

    def rows(self, first=0, count=None, with_sax=True):
        count = self.n - first if count is None else count
        rows = np.zeros((count, self.L), dtype=np.float32)
        sax = np.zeros((count, 16), dtype=np.uint8) if with_sax else None
        _check(lib().hg_index_rows(self._h, first, count, _ptr(rows), _ptr(sax)))
        return (rows, sax) if with_sax else rows

    # -- queries -------------------------------------------------------------
    def knn(self, queries, k=1, mode=MODE_PLAIN, use_lb_sax=False, with_leaf_pos=False, stats=False,
            profile=False, epsilon=0.0, nprobes=0, approx_leaves=0):
        """Exact k-NN (squared distances ascending, dataset ids); epsilon > 0
        or nprobes > 0 give the reference's epsilon-approximate or nprobes
        search instead; approx_leaves > 1 seeds the exact search with that
        many leaves best-first (the answers are the same)."""
        q = _f32(queries, self.L)
        nq = q.shape[0]
        d = np.zeros((nq, k), dtype=np.float32)
        ids = np.zeros((nq, k), dtype=np.int64)
        pos = np.zeros((nq, k), dtype=np.uint64) if with_leaf_pos else None
        st = QueryStats()
        opts = KnnOpts(mode, 1 if use_lb_sax else 0, 1 if profile else 0, 0, 0, 0, float(epsilon), int(nprobes),
                       int(approx_leaves))
        _check(lib().hg_knn(self._h, _ptr(q), nq, k, ctypes.byref(opts), _ptr(d), _ptr(ids), _ptr(pos),
                            ctypes.byref(st)))
        out = [d, ids]
        if with_leaf_pos:
            out.append(pos)
        if stats:
            out.append(st.as_dict())
        return tuple(out)

    def pscan(self, queries, k=1, stats=False):
        return self.knn(queries, k, mode=MODE_PSCAN, stats=stats)

    def knn_device(self, q_ptr, nq, k, dist_ptr, id_ptr, stream=0, mode=MODE_PLAIN, use_lb_sax=False,
                   profile=False, approx_leaves=0):
        """Device-resident variant; pointers are raw device addresses."""
        st = QueryStats()
        opts = KnnOpts(mode, 1 if use_lb_sax else 0, 1 if profile else 0, 0, 0, 0, 0.0, 0, int(approx_leaves))
        _check(lib().hg_knn_device(self._h, ctypes.c_void_p(q_ptr), nq, k, ctypes.byref(opts),
                                   ctypes.c_void_p(dist_ptr), ctypes.c_void_p(id_ptr), ctypes.c_void_p(stream),
                                   ctypes.byref(st)))
        return st.as_dict()

    def knn_batch(self, queries, k, stats=False, bucket_cap=0, dense_filter=False):
        """Batched exact k-NN (BF16 tensor-core filter + exact re-rank); k is
        an int or one k per query.  Outputs are nq x max(k); entries past a
        query's k are +inf / -1.  dense_filter: filter every row against every
        query (no LB_EAPCA leaf pruning first); the answers are the same."""
        q = _f32(queries, self.L)
        nq = q.shape[0]
        ks = np.broadcast_to(np.asarray(k, dtype=np.uint32), (nq,)).copy()
        kmax = int(ks.max()) if nq else int(np.max(k))
        d = np.zeros((nq, kmax), dtype=np.float32)
        ids = np.zeros((nq, kmax), dtype=np.int64)
        st = QueryStats()
        opts = KnnOpts(MODE_BATCH, 1, 0, 0, bucket_cap, int(bool(dense_filter)))
        _check(lib().hg_knn_batch(self._h, _ptr(q), nq, _ptr(ks), kmax, ctypes.byref(opts), _ptr(d), _ptr(ids),
                                  ctypes.byref(st)))
        return (d, ids, st.as_dict()) if stats else (d, ids)

    def knn_batch_device(self, q_ptr, nq, ks, kmax, dist_ptr, id_ptr, stream=0, bucket_cap=0, dense_filter=False):
        """Device-resident batched variant; ks is a host array (or None)."""
        st = QueryStats()
        opts = KnnOpts(MODE_BATCH, 1, 0, 0, bucket_cap, int(bool(dense_filter)))
        kp = None
        if ks is not None:
            ks = np.ascontiguousarray(ks, dtype=np.uint32)
            kp = _ptr(ks)
        _check(lib().hg_knn_batch_device(self._h, ctypes.c_void_p(q_ptr), nq, kp, kmax, ctypes.byref(opts),
                                         ctypes.c_void_p(dist_ptr), ctypes.c_void_p(id_ptr),
                                         ctypes.c_void_p(stream), ctypes.byref(st)))
        return st.as_dict()

    def tuning(self):
        t = Tuning()
        _check(lib().hg_tuning_get(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = Tuning(**kw)
        _check(lib().hg_tuning_set(self._h, ctypes.byref(t)))

    def autotune_device(self, q_ptr, nq, ks, kmax, stream=0):
        """Times candidate launch parameters on device queries and keeps the fastest."""
        t = Tuning()
        kp = None
        if ks is not None:
            ks = np.ascontiguousarray(ks, dtype=np.uint32)
            kp = _ptr(ks)
        _check(lib().hg_autotune(self._h, ctypes.c_void_p(q_ptr), nq, kp, kmax, ctypes.c_void_p(stream),
                                 ctypes.byref(t)))
        return t.as_dict()

    def route(self, queries):
        q = _f32(queries, self.L)
        out = np.zeros(q.shape[0], dtype=np.int32)
        _check(lib().hg_route(self._h, _ptr(q), q.shape[0], _ptr(out)))
        return out

    def leaf_lower_bounds(self, query):
        q = _f32(query).reshape(-1)
        out = np.zeros(self.info.num_leaves, dtype=np.float32)
        _check(lib().hg_leaf_lower_bounds(self._h, _ptr(q), _ptr(out)))
        return out


def bf16_dots_device(rows_ptr, n, L, q_ptr, nq, out_ptr, stream=0):
    """Tensor-core products q~.x~ of the batched filter (diagnostics)."""
    _check(lib().hg_bf16_dots(ctypes.c_void_p(rows_ptr), n, L, ctypes.c_void_p(q_ptr), nq, ctypes.c_void_p(out_ptr),
                              ctypes.c_void_p(stream)))


# -- data --------------------------------------------------------------------

def filter_wait_check(wait_us, withhold, stream=0):
    """hg_filter_wait_check: the status code (HG_OK, or HG_ERR_TIMEOUT when a
    withheld copy makes the filter kernel's shortened wait run out)."""
    return lib().hg_filter_wait_check(wait_us, int(bool(withhold)), ctypes.c_void_p(stream))


def filter_pair_wait_check(wait_us, withhold, stream=0):
    """hg_filter_pair_wait_check: the same for the CTA-pair filter kernel."""
    return lib().hg_filter_pair_wait_check(wait_us, int(bool(withhold)), ctypes.c_void_p(stream))


def generate_walks(seed, n, L, first=0):
    """Host-side z-normalised random walks (same bits as the GPU generator)."""
    out = np.zeros((n, L), dtype=np.float32)
    _check(lib().hg_generate_walks(seed, first, n, L, _ptr(out), 0, 0))
    return out


def generate_walks_device(seed, n, L, out_ptr, first=0, device=0):
    _check(lib().hg_generate_walks(seed, first, n, L, ctypes.c_void_p(out_ptr), 1, device))


def generate_queries(seed, data, sigma2, return_base=False):
    data = _f32(data)
    n, L = data.shape
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    nq = s2.shape[0]
    out = np.zeros((nq, L), dtype=np.float32)
    base = np.zeros(nq, dtype=np.uint64)
    _check(lib().hg_generate_queries(seed, _ptr(data), n, L, nq, _ptr(s2), _ptr(out), _ptr(base), 0, 0))
    return (out, base) if return_base else out


def generate_queries_device(seed, data_ptr, n, L, sigma2, out_ptr, base_ptr=None, device=0):
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    _check(lib().hg_generate_queries(seed, ctypes.c_void_p(data_ptr), n, L, s2.shape[0], _ptr(s2),
                                     ctypes.c_void_p(out_ptr), ctypes.c_void_p(base_ptr) if base_ptr else None,
                                     1, device))


def generate_unit_vectors(seed, n, L, first=0):
    """Host-side unit-normalised Gaussian rows (same bits as the GPU generator)."""
    out = np.zeros((n, L), dtype=np.float32)
    _check(lib().hg_generate_unit_vectors(seed, first, n, L, _ptr(out), 0, 0))
    return out


def generate_unit_vectors_device(seed, n, L, out_ptr, first=0, device=0):
    _check(lib().hg_generate_unit_vectors(seed, first, n, L, ctypes.c_void_p(out_ptr), 1, device))


def generate_unit_queries(seed, data, sigma2):
    data = _f32(data)
    n, L = data.shape
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    out = np.zeros((s2.shape[0], L), dtype=np.float32)
    _check(lib().hg_generate_unit_queries(seed, _ptr(data), n, L, s2.shape[0], _ptr(s2), _ptr(out), None, 0, 0))
    return out


def generate_unit_queries_device(seed, data_ptr, n, L, sigma2, out_ptr, device=0):
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    _check(lib().hg_generate_unit_queries(seed, ctypes.c_void_p(data_ptr), n, L, s2.shape[0], _ptr(s2),
                                          ctypes.c_void_p(out_ptr), None, 1, device))


def generate_queries_seeded(data_seed, seed, n, L, sigma2, unit=False, return_base=False):
    """Noisy queries over the seeded collection of data_seed (n rows), base
    rows regenerated on the host: the bits of generate_queries /
    generate_unit_queries given that collection."""
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    out = np.zeros((s2.shape[0], L), dtype=np.float32)
    base = np.zeros(s2.shape[0], dtype=np.uint64)
    _check(lib().hg_generate_queries_seeded(data_seed, seed, n, L, s2.shape[0], _ptr(s2), int(bool(unit)),
                                            _ptr(out), _ptr(base), 0, 0))
    return (out, base) if return_base else out


def generate_queries_seeded_device(data_seed, seed, n, L, sigma2, out_ptr, unit=False, device=0):
    s2 = np.ascontiguousarray(sigma2, dtype=np.float64)
    _check(lib().hg_generate_queries_seeded(data_seed, seed, n, L, s2.shape[0], _ptr(s2), int(bool(unit)),
                                            ctypes.c_void_p(out_ptr), None, 1, device))


def sax_breakpoints():
    out = np.zeros(255, dtype=np.float32)
    _check(lib().hg_sax_breakpoints(_ptr(out)))
    return out


def pscan_noalloc(rows_ptr, n, L, query_ptr, k, dist_ptr, id_ptr, stream=0):
    """Allocation-free exact k-NN scan of a caller-owned device matrix
    (hg_pscan_noalloc); all pointers are device addresses."""
    _check(lib().hg_pscan_noalloc(ctypes.c_void_p(rows_ptr), n, L, ctypes.c_void_p(query_ptr), k,
                                  ctypes.c_void_p(dist_ptr), ctypes.c_void_p(id_ptr), ctypes.c_void_p(stream)))
