"""Parity checker for hercules_b200 -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
--impl reference legs may import this module.  It wraps

  _build/liboracle.so      the CPU restatement of the reference's exact k-NN
                           path (hercules_oracle.c), plain C, no fused
                           multiply-adds;
  _ref/libref_hercules.so  the reference's own library sources compiled here
                           (Makefile target `ref`) plus ref_shim.c, to pin
                           the restatement bit for bit;
  _ref/hercules, _ref/hercules_nofma, _ref/pscan
                           the reference command lines built from source;

and an FP64 brute force.
"""
import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SO = os.path.join(REF_DIR, "libref_hercules.so")
REF_BIN = os.path.join(REF_DIR, "hercules")
REF_BIN_NOFMA = os.path.join(REF_DIR, "hercules_nofma")
REF_PSCAN = os.path.join(REF_DIR, "pscan")
# Where the reference's sources lie: HERCULES_REF, else the conventional
# read-only checkout path of the build container (absent on other machines,
# where only the prebuilt _ref/ files are used).
REFERENCE_ROOT = os.environ.get("HERCULES_REF") or "/root/reference"


def have_ref_sources():
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "code", "hercules"))

_P = ctypes.c_void_p


def build(ref=None):
    """Compile the restatement (and the reference when its sources exist)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    if ref is None:
        ref = have_ref_sources()
    if ref:
        subprocess.run(["make", "-s", "-C", HERE, "ref", "REF=" + REFERENCE_ROOT], check=True)


def have_ref():
    return os.path.exists(REF_SO) and os.path.exists(REF_BIN)


class _Stats(ctypes.Structure):
    _fields_ = [("loaded_leaves", ctypes.c_uint32), ("loaded_rows", ctypes.c_uint64),
                ("candidate_leaves", ctypes.c_uint32), ("approx_leaf", ctypes.c_uint32)]


_o = None
_r = None


def olib():
    global _o
    if _o is None:
        if not os.path.exists(ORACLE_SO):
            build(ref=False)
        L = ctypes.CDLL(ORACLE_SO)
        f32, i32, u32, u64, i64 = ctypes.c_float, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int64
        sig = {
            "or_ed": (f32, [_P, _P, i32, f32]),
            "or_mean_stdev": (None, [_P, i32, i32, _P, _P]),
            "or_paa": (None, [_P, _P, i32]),
            "or_sax": (None, [_P, _P, i32, _P]),
            "or_lb_sax": (f32, [_P, _P, i32, _P]),
            "or_lb_eapca": (f32, [_P, i32, _P, _P]),
            "or_topk_insert": (None, [_P, _P, _P, _P, i32, f32, i64, u64, i32]),
            "or_build": (_P, [_P, u64, i32, i32]),
            "or_build_mt": (_P, [_P, u64, i32, i32, i32, i32]),
            "or_gen_rows": (None, [u64, u64, u64, i32, _P, i32, i32]),
            "or_gen_queries": (None, [u64, u64, u64, i32, i32, _P, _P, _P, i32]),
            "or_write": (i32, [_P, ctypes.c_char_p, ctypes.c_double, _P]),
            "or_read": (_P, [ctypes.c_char_p]),
            "or_free": (None, [_P]),
            "or_num_leaves": (i32, [_P]),
            "or_num_nodes": (i32, [_P]),
            "or_L": (i32, [_P]),
            "or_num_rows": (u64, [_P]),
            "or_leaf_info": (None, [_P, i32, _P, _P, _P, _P, _P]),
            "or_row_ids": (None, [_P, _P]),
            "or_rows": (_P, [_P]),
            "or_exact_knn": (i32, [_P, _P, i32, i32, _P, _P, _P, ctypes.POINTER(_Stats)]),
            "or_approx_knn": (i32, [_P, _P, i32, i32, ctypes.c_float, i32, _P, _P, _P, ctypes.POINTER(_Stats)]),
            "or_leaf_lbs": (None, [_P, _P, _P]),
            "or_pscan": (i32, [_P, u64, i32, _P, i32, i32, _P, _P]),
        }
        for k, (res, args) in sig.items():
            fn = getattr(L, k)
            fn.restype = res
            fn.argtypes = args
        _o = L
    return _o


def rlib():
    """The reference primitives (compiled from the reference sources)."""
    global _r
    if _r is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("reference library not built (make -C oracle ref)")
        L = ctypes.CDLL(REF_SO)
        f32, i32 = ctypes.c_float, ctypes.c_int
        sig = {
            "shim_ed": (f32, [_P, _P, i32, f32]),
            "shim_mean_stdev": (None, [_P, i32, i32, _P, _P]),
            "shim_paa": (None, [_P, _P, i32]),
            "shim_sax": (None, [_P, _P, i32]),
            "shim_lb_sax": (f32, [_P, _P, i32]),
            "shim_lb_eapca": (f32, [_P, i32, _P, _P]),
            "shim_topk_insert": (None, [_P, _P, _P, ctypes.c_uint, f32, ctypes.c_longlong]),
            "shim_breakpoints": (None, [_P]),
        }
        for k, (res, args) in sig.items():
            fn = getattr(L, k)
            fn.restype = res
            fn.argtypes = args
        _r = L
    return _r


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


GOLDEN_BP = os.path.join(os.path.dirname(HERE), "tests", "golden", "sax_breakpoints_card256.txt")


def breakpoints():
    """The reference's 255 breakpoints of cardinality 256 (golden fixture)."""
    return np.loadtxt(GOLDEN_BP, dtype=np.float64).astype(np.float32)


# ---- primitives -------------------------------------------------------------

def ed(q, x, bound=np.inf):
    q = np.ascontiguousarray(q, np.float32)
    x = np.ascontiguousarray(x, np.float32)
    return olib().or_ed(_p(q), _p(x), q.shape[0], float(np.float32(bound)))


def mean_stdev(x, start, end):
    x = np.ascontiguousarray(x, np.float32)
    m, s = ctypes.c_float(), ctypes.c_float()
    olib().or_mean_stdev(_p(x), start, end, ctypes.byref(m), ctypes.byref(s))
    return np.float32(m.value), np.float32(s.value)


def paa(ts):
    ts = np.ascontiguousarray(ts, np.float32)
    out = np.zeros(16, np.float32)
    olib().or_paa(_p(ts), _p(out), ts.shape[0])
    return out


def sax(ts, bp=None):
    ts = np.ascontiguousarray(ts, np.float32)
    bp = breakpoints() if bp is None else np.ascontiguousarray(bp, np.float32)
    out = np.zeros(16, np.uint8)
    olib().or_sax(_p(ts), _p(out), ts.shape[0], _p(bp))
    return out


def lb_sax(paa_q, word, L, bp=None):
    bp = breakpoints() if bp is None else np.ascontiguousarray(bp, np.float32)
    return olib().or_lb_sax(_p(np.ascontiguousarray(paa_q, np.float32)), _p(np.ascontiguousarray(word, np.uint8)),
                            L, _p(bp))


def lb_eapca(q, points, sk):
    q = np.ascontiguousarray(q, np.float32)
    pts = np.ascontiguousarray(points, np.int16)
    sk = np.ascontiguousarray(sk, np.float32)
    return olib().or_lb_eapca(_p(q), pts.shape[0], _p(pts), _p(sk))


# ---- index ----------------------------------------------------------------

class OracleIndex:
    def __init__(self, handle, keep=None):
        self.h = ctypes.c_void_p(handle)
        self._keep = keep

    @classmethod
    def build(cls, data, leaf_size):
        data = np.ascontiguousarray(data, np.float32)
        h = olib().or_build(_p(data), data.shape[0], data.shape[1], leaf_size)
        if not h:
            raise ValueError("or_build failed")
        return cls(h, data)

    @classmethod
    def build_mt(cls, data, leaf_size, threads=0, keep_rows=True):
        """or_build on several threads (same index).  keep_rows=False keeps
        no leaf-ordered copy: such an index can only be written."""
        data = np.ascontiguousarray(data, np.float32)
        h = olib().or_build_mt(_p(data), data.shape[0], data.shape[1], leaf_size, int(threads), int(bool(keep_rows)))
        if not h:
            raise ValueError("or_build_mt failed")
        return cls(h, data)

    @classmethod
    def read(cls, directory):
        if not directory.endswith("/"):
            directory += "/"
        h = olib().or_read(directory.encode())
        if not h:
            raise IOError("or_read failed for " + directory)
        return cls(h)

    def write(self, directory, buffer_mb=0.0):
        if not directory.endswith("/"):
            directory += "/"
        bp = breakpoints()
        if olib().or_write(self.h, directory.encode(), float(buffer_mb), _p(bp)) != 0:
            raise IOError("or_write failed")

    def __del__(self):
        if getattr(self, "h", None):
            olib().or_free(self.h)
            self.h = None

    @property
    def L(self):
        return olib().or_L(self.h)

    @property
    def n(self):
        return olib().or_num_rows(self.h)

    def num_leaves(self):
        return olib().or_num_leaves(self.h)

    def leaves(self):
        out = []
        for i in range(self.num_leaves()):
            fp, sz, ns = ctypes.c_uint64(), ctypes.c_uint32(), ctypes.c_int()
            olib().or_leaf_info(self.h, i, ctypes.byref(fp), ctypes.byref(sz), ctypes.byref(ns), None, None)
            out.append((fp.value, sz.value, ns.value))
        return out

    def leaf_envelope(self, i):
        ns = self.leaves()[i][2]
        pts = np.zeros(ns, np.int16)
        sk = np.zeros((ns, 4), np.float32)
        olib().or_leaf_info(self.h, i, None, None, None, _p(pts), _p(sk))
        return pts, sk

    def row_ids(self):
        ids = np.zeros(self.n, np.int64)
        olib().or_row_ids(self.h, _p(ids))
        return ids

    def rows(self):
        ptr = olib().or_rows(self.h)
        n, L = self.n, self.L
        return np.ctypeslib.as_array(ctypes.cast(ptr, ctypes.POINTER(ctypes.c_float)), shape=(n, L)).copy()

    def knn(self, q, k=1, tie_lowest=True):
        """exact_de_knn_search: (squared distances, leaf-ordered rows, leaf file_pos, stats)."""
        q = np.ascontiguousarray(q, np.float32)
        d = np.zeros(k, np.float32)
        rows = np.zeros(k, np.int64)
        fp = np.zeros(k, np.uint64)
        st = _Stats()
        olib().or_exact_knn(self.h, _p(q), k, 1 if tie_lowest else 0, _p(d), _p(rows), _p(fp), ctypes.byref(st))
        return d, rows, fp, {f: getattr(st, f) for f, _ in st._fields_}

    def approx_knn(self, q, k=1, epsilon=0.0, nprobes=0, tie_lowest=True):
        """exact_de_knn_search with epsilon, or exact_ng_knn_search with nprobes:
        (squared distances, leaf-ordered rows, leaf file_pos, stats)."""
        q = np.ascontiguousarray(q, np.float32)
        d = np.zeros(k, np.float32)
        rows = np.zeros(k, np.int64)
        fp = np.zeros(k, np.uint64)
        st = _Stats()
        olib().or_approx_knn(self.h, _p(q), k, 1 if tie_lowest else 0, float(epsilon), int(nprobes), _p(d),
                             _p(rows), _p(fp), ctypes.byref(st))
        return d, rows, fp, {f: getattr(st, f) for f, _ in st._fields_}

    def leaf_lbs(self, q):
        q = np.ascontiguousarray(q, np.float32)
        out = np.zeros(self.num_leaves(), np.float32)
        olib().or_leaf_lbs(self.h, _p(q), _p(out))
        return out


def gen_rows(seed, n, L, first=0, unit=False, threads=0, out=None):
    """Rows [first, first+n) of the seeded generator (random walks, or unit
    vectors with unit=True): the same bits as hercules_b200's generator."""
    if out is None:
        out = np.empty((n, L), np.float32)
    olib().or_gen_rows(seed, first, n, L, _p(out), int(bool(unit)), int(threads))
    return out


def gen_queries(data_seed, seed, n, L, sigma2, unit=False):
    """Noisy queries over a collection of n rows of stream data_seed (row
    pick(j) plus N(0, sigma2[j]) noise, normalised); returns (queries, base
    row ids)."""
    s2 = np.ascontiguousarray(sigma2, np.float64)
    nq = s2.shape[0]
    out = np.empty((nq, L), np.float32)
    base = np.empty(nq, np.uint64)
    olib().or_gen_queries(data_seed, seed, n, L, nq, _p(s2), _p(out), _p(base), int(bool(unit)))
    return out, base


def pscan(data, q, k=1, tie_lowest=True):
    data = np.ascontiguousarray(data, np.float32)
    q = np.ascontiguousarray(q, np.float32)
    d = np.zeros(k, np.float32)
    ids = np.zeros(k, np.int64)
    olib().or_pscan(_p(data), data.shape[0], data.shape[1], _p(q), k, 1 if tie_lowest else 0, _p(d), _p(ids))
    return d, ids


def brute_force_fp64(data, queries, k):
    """FP64 exact k-NN (squared distances and ids), for error reporting."""
    data64 = np.asarray(data, np.float64)
    out_d, out_i = [], []
    n2 = (data64 * data64).sum(1)
    for q in np.asarray(queries, np.float64).reshape(-1, data64.shape[1]):
        d = n2 - 2.0 * data64 @ q + (q * q).sum()
        idx = np.argpartition(d, min(k, len(d) - 1))[: k + 8]
        # exact recomputation for the short list
        dd = ((data64[idx] - q) ** 2).sum(1)
        o = np.lexsort((idx, dd))[:k]
        out_d.append(dd[o])
        out_i.append(idx[o])
    return np.array(out_d), np.array(out_i)


# ---- the reference command line ----------------------------------------------

def ref_build_index(binary, dataset, n, L, leaf, index_dir, buffer_mb=None, threads=2):
    """Reference build: --mode 0 --serial 1 --sims with one insert worker."""
    if buffer_mb is None:
        # room for the data and every split's copy, so that no flush happens
        buffer_mb = max(64.0, n * L * 4 * 12 / 2 ** 20)
    if not index_dir.endswith("/"):
        index_dir += "/"
    cmd = [binary, "--mode", "0", "--serial", "1", "--sims", "--num-threads", str(threads), "--num-write-threads",
           "1", "--initial-db-size", "120000", "--buffer-size", str(buffer_mb), "--leaf-size", str(leaf),
           "--timeseries-size", str(L), "--dataset-size", str(n), "--dataset", dataset, "--index-path", index_dir]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=3600)
    if r.returncode != 0:
        raise RuntimeError("reference build failed: %s" % r.stderr[-2000:])
    return buffer_mb


_TSV = re.compile(r"^(Query_[A-Za-z_]+)\t([^\t]*)\t([^\t]*)\t(\d+)\t(\d+)$")


def ref_query(binary, index_dir, queries_file, nq, k, threads=1, extra=()):
    """Reference query run; returns {field: array[nq, k]} parsed from the TSV."""
    if not index_dir.endswith("/"):
        index_dir += "/"
    cmd = [binary, "--mode", "1", "--serial", "1", "--num-threads", str(threads), "--k", str(k), "--queries",
           queries_file, "--queries-size", str(nq), "--index-path", index_dir, *extra]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=7200, cwd=index_dir)
    if r.returncode != 0:
        raise RuntimeError("reference query failed: %s" % r.stderr[-2000:])
    fields = {}
    for line in r.stdout.splitlines():
        m = _TSV.match(line)
        if not m:
            continue
        name, val, _qf, qn, rank = m.groups()
        fields.setdefault(name, {})[(int(qn), int(rank))] = val
    out = {}
    for name, d in fields.items():
        arr = np.full((nq, k), np.nan, dtype=object)
        for (qn, rank), v in d.items():
            if 1 <= qn <= nq and 1 <= rank <= k:
                arr[qn - 1, rank - 1] = v
        out[name] = arr
    return out


def parse_root_idx(path):
    """Parse root.idx into (header, [node records]); the 28 trailing bytes of
    each raw struct node_split_policy (padding and heap pointers, not
    meaningful) are dropped so that two files compare field by field."""
    import struct
    b = open(path, "rb").read()
    hdr = struct.unpack_from("<QdIIiiIii", b, 0)
    off = struct.calcsize("<QdIIiiIii")
    nodes = []

    def node():
        nonlocal off
        is_leaf, level = struct.unpack_from("<BI", b, off)
        off += 5
        rec = {"is_leaf": is_leaf, "level": level}
        if not is_leaf:
            node()
            node()
            size, split_seg = struct.unpack_from("<Ih", b, off)
            off += 6
            pol = b[off:off + 20]
            off += 48
            rec.update(size=size, split_segment=split_seg, policy=pol)
        else:
            size, flen = struct.unpack_from("<Ii", b, off)
            off += 8
            rec.update(size=size, filename=b[off:off + max(flen, 0)].decode())
            off += max(flen, 0)
            if flen <= 0:
                nodes.append(rec)
                return
        (np_,) = struct.unpack_from("<h", b, off)
        off += 2
        rec["points"] = list(struct.unpack_from("<%dh" % np_, b, off))
        off += 2 * np_
        sk = []
        for _ in range(np_):
            (ni,) = struct.unpack_from("<i", b, off)
            off += 4
            sk.append(b[off:off + 4 * ni])
            off += 4 * ni
        rec["sketch"] = sk
        if is_leaf:
            (rec["file_pos"],) = struct.unpack_from("<Q", b, off)
            off += 8
        nodes.append(rec)

    node()
    assert off == len(b), (off, len(b))
    return hdr, nodes
