"""Generates the golden fixtures of tests/golden from the reference itself.

Run in a container that has the reference sources (it compiles them with
oracle/Makefile `ref`); the GPU box only reads the committed outputs.

  sax_breakpoints_card256.txt  the reference's 255 breakpoints of cardinality
                               256 (include/sax_breakpoints.h, offset 32385)
  kat_primitives.npz           inputs and the reference library's outputs for
                               the distance, mean/stdev, PAA, iSAX, LB_SAX,
                               LB_EAPCA and top-k insert primitives
  ref_<config>.json            for seeded datasets: SHA-256 of the dataset,
                               of the reference's leaves_raw.idx and
                               leaves_sims.idx and of its root.idx fields;
                               the reference CLI's answers (Query_exact_*)
                               and per-query load counters, exact and with
                               --epsilon 0.5 / 2 and --nprobes 3 / 10
  ref_walks1M_L256_leaf100000.json
                               the plain method's CPU-runnable configuration:
                               1M z-normalised random walks of length 256
                               (seed 1184), leaf size 100,000, 100 fresh
                               random-walk queries (seed 14784) answered one
                               at a time with k = 1 and k = 10: index digests
                               and the reference CLI's answers and counters

Usage: python tests/golden/make_golden.py [all | config1]
"""
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
import hercules_b200 as H  # noqa: E402

CONFIGS = [
    # name, n, L, leaf, queries, k
    ("n20000_L64_leaf500", 20000, 64, 500, 30, 10),
    ("n100000_L256_leaf2000", 100000, 256, 2000, 30, 10),
    ("n30000_L96_leaf700", 30000, 96, 700, 20, 5),
]
DATA_SEED = 1184
QUERY_SEED = 14784
APPROX_MODES = [("eps0.5", ("--epsilon", "0.5")), ("eps2", ("--epsilon", "2")),
                ("np3", ("--nprobes", "3")), ("np10", ("--nprobes", "10"))]


def sha(b):
    return hashlib.sha256(b).hexdigest()


def root_fields_digest(path):
    hdr, nodes = O.parse_root_idx(path)
    h = hashlib.sha256(repr(hdr).encode())
    for rec in nodes:
        h.update(repr(sorted((k, v.hex() if isinstance(v, bytes) else
                              [x.hex() for x in v] if k == "sketch" else v) for k, v in rec.items())).encode())
    return h.hexdigest()


def breakpoints():
    s = open(os.path.join(O.REFERENCE_ROOT, "code/hercules/include/sax_breakpoints.h")).read()
    vals = [v.strip() for v in s[s.index("{") + 1:s.index("}")].split(",")][32385:32385 + 255]
    with open(os.path.join(HERE, "sax_breakpoints_card256.txt"), "w") as f:
        f.write("# sax_breakpoints[32385..32639] of code/hercules/include/sax_breakpoints.h (cardinality 256)\n")
        f.write("\n".join(vals) + "\n")


def kat_primitives():
    import ctypes
    r = O.rlib()
    rng = np.random.default_rng(5)
    out = {}
    for L in (64, 256):
        X = H.generate_walks(77, 24, L)
        Q = H.generate_walks(78, 8, L)
        bounds = np.array([np.inf, 40.0, 150.0], np.float32)
        ed = np.zeros((8, 24, 3), np.float32)
        for i, q in enumerate(Q):
            for j, x in enumerate(X):
                for b, bd in enumerate(bounds):
                    ed[i, j, b] = r.shim_ed(O._p(q), O._p(x), L, bd)
        segs = np.array([(0, L), (0, L // 2), (3, 17), (L // 3, L - 1), (5, 6), (L - 9, L)], np.int32)
        ms = np.zeros((8, len(segs), 2), np.float32)
        for i, q in enumerate(Q):
            for s, (a, b) in enumerate(segs):
                m, sd = ctypes.c_float(), ctypes.c_float()
                r.shim_mean_stdev(O._p(q), int(a), int(b), ctypes.byref(m), ctypes.byref(sd))
                ms[i, s] = (m.value, sd.value)
        paa = np.zeros((8, 16), np.float32)
        for i, q in enumerate(Q):
            r.shim_paa(O._p(q), O._p(paa[i]), L)
        words = np.zeros((24, 16), np.uint8)
        for j, x in enumerate(X):
            r.shim_sax(O._p(x), O._p(words[j]), L)
        lbsax = np.zeros((8, 24), np.float32)
        for i in range(8):
            for j in range(24):
                lbsax[i, j] = r.shim_lb_sax(O._p(paa[i]), O._p(words[j]), L)
        pts_l, sk_l, lb_l = [], [], []
        for t in range(16):
            nseg = int(rng.integers(1, 9))
            pts = np.array(sorted(rng.choice(np.arange(1, L), nseg - 1, replace=False).tolist()) + [L], np.int16)
            sk = np.zeros((nseg, 4), np.float32)
            for s in range(nseg):
                a, b = np.sort(rng.normal(size=2)).astype(np.float32)
                c, d = np.sort(np.abs(rng.normal(size=2))).astype(np.float32)
                sk[s] = [b, a, d, c]
            pad_p = np.zeros(8, np.int16)
            pad_p[:nseg] = pts
            pad_s = np.zeros((8, 4), np.float32)
            pad_s[:nseg] = sk
            pts_l.append(pad_p)
            sk_l.append(pad_s)
            lb_l.append([r.shim_lb_eapca(O._p(Q[i]), nseg, O._p(pts), O._p(sk)) for i in range(8)])
        out.update({f"L{L}_X": X, f"L{L}_Q": Q, f"L{L}_bounds": bounds, f"L{L}_ed": ed, f"L{L}_segs": segs,
                    f"L{L}_ms": ms, f"L{L}_paa": paa, f"L{L}_sax": words, f"L{L}_lbsax": lbsax,
                    f"L{L}_eapca_points": np.array(pts_l), f"L{L}_eapca_sk": np.array(sk_l),
                    f"L{L}_eapca_lb": np.array(lb_l, np.float32)})
    # top-k insert sequences with duplicates
    seq = np.array([5, 3, 3, 9, 1, 5, 2, 2, 0.5, 7, 1, 4], np.float32)
    for k in (1, 3, 5):
        dist = np.full(k, np.finfo(np.float32).max, np.float32)
        ids = np.full(k, -1, np.int64)
        cur = ctypes.c_uint(0)
        for i, d in enumerate(seq):
            if d < dist[k - 1]:
                r.shim_topk_insert(O._p(dist), O._p(ids), ctypes.byref(cur), k, d, i)
        out[f"topk_k{k}_dist"] = dist.copy()
        out[f"topk_k{k}_ids"] = ids.copy()
    out["topk_seq"] = seq
    np.savez_compressed(os.path.join(HERE, "kat_primitives.npz"), **out)


def ref_config(name, n, L, leaf, nq, k):
    tmp = tempfile.mkdtemp(prefix="golden_")
    try:
        X = H.generate_walks(DATA_SEED, n, L)
        X.tofile(os.path.join(tmp, "data.bin"))
        s2 = np.array([0.01, 0.1, 1.0] * nq)[:nq]
        Q = H.generate_queries(QUERY_SEED, X, s2)
        Q.tofile(os.path.join(tmp, "q.bin"))
        res = {"n": n, "L": L, "leaf": leaf, "nq": nq, "k": k, "data_seed": DATA_SEED, "query_seed": QUERY_SEED,
               "sigma2": s2.tolist(), "data_sha256": sha(X.tobytes()), "queries_sha256": sha(Q.tobytes()),
               "buffer_mb": 500.0}
        for tag, binary in (("stock", O.REF_BIN), ("nofma", O.REF_BIN_NOFMA)):
            d = os.path.join(tmp, tag) + "/"
            O.ref_build_index(binary, os.path.join(tmp, "data.bin"), n, L, leaf, d, buffer_mb=500.0)
            res[tag] = {
                "leaves_raw_sha256": sha(open(d + "leaves_raw.idx", "rb").read()),
                "leaves_sims_sha256": sha(open(d + "leaves_sims.idx", "rb").read()),
                "root_fields_sha256": root_fields_digest(d + "root.idx"),
            }
            if tag == "stock":
                q = O.ref_query(binary, d, os.path.join(tmp, "q.bin"), nq, k)
                res["answers"] = {
                    "exact_distance": q["Query_exact_distance"].tolist(),
                    "exact_node_file_pos": q["Query_exact_node_file_pos"].tolist(),
                    "loaded_nodes": q["Query_total_loaded_nodes_count"][:, 0].tolist(),
                    "loaded_ts": q["Query_total_loaded_ts_count"][:, 0].tolist(),
                }
                # the approximate searches of the same serial path
                res["approx"] = {}
                for mode, extra in APPROX_MODES:
                    qa = O.ref_query(binary, d, os.path.join(tmp, "q.bin"), nq, k, extra=extra)
                    res["approx"][mode] = {
                        "args": list(extra),
                        "exact_distance": qa["Query_exact_distance"].tolist(),
                        "exact_node_file_pos": qa["Query_exact_node_file_pos"].tolist(),
                    }
                hdr, nodes = O.parse_root_idx(d + "root.idx")
                res["num_leaves"] = hdr[0]
                res["num_nodes"] = len(nodes)
        with open(os.path.join(HERE, f"ref_{name}.json"), "w") as f:
            json.dump(res, f, indent=1)
    finally:
        shutil.rmtree(tmp)


CONFIG1 = ("walks1M_L256_leaf100000", 1000000, 256, 100000, 100, (1, 10))


def ref_config1(name, n, L, leaf, nq, ks):
    """1M x 256 walks, leaf 100,000; queries are fresh random walks of the
    query seed (the same generator, an independent seed)."""
    tmp = tempfile.mkdtemp(prefix="golden_")
    try:
        X = H.generate_walks(DATA_SEED, n, L)
        X.tofile(os.path.join(tmp, "data.bin"))
        Q = H.generate_walks(QUERY_SEED, nq, L)
        Q.tofile(os.path.join(tmp, "q.bin"))
        buffer_mb = 4096.0  # holds the data and every split's copy: no flush
        res = {"n": n, "L": L, "leaf": leaf, "nq": nq, "ks": list(ks), "data_seed": DATA_SEED,
               "query_seed": QUERY_SEED, "queries": "fresh random walks", "data_sha256": sha(X.tobytes()),
               "queries_sha256": sha(Q.tobytes()), "buffer_mb": buffer_mb}
        d = os.path.join(tmp, "stock") + "/"
        O.ref_build_index(O.REF_BIN, os.path.join(tmp, "data.bin"), n, L, leaf, d, buffer_mb=buffer_mb)
        res["stock"] = {
            "leaves_raw_sha256": sha(open(d + "leaves_raw.idx", "rb").read()),
            "leaves_sims_sha256": sha(open(d + "leaves_sims.idx", "rb").read()),
            "root_fields_sha256": root_fields_digest(d + "root.idx"),
        }
        hdr, nodes = O.parse_root_idx(d + "root.idx")
        res["num_leaves"] = hdr[0]
        res["num_nodes"] = len(nodes)
        res["answers"] = {}
        for k in ks:
            q = O.ref_query(O.REF_BIN, d, os.path.join(tmp, "q.bin"), nq, k)
            res["answers"]["k%d" % k] = {
                "exact_distance": q["Query_exact_distance"].tolist(),
                "exact_node_file_pos": q["Query_exact_node_file_pos"].tolist(),
                "loaded_nodes": q["Query_total_loaded_nodes_count"][:, 0].tolist(),
                "loaded_ts": q["Query_total_loaded_ts_count"][:, 0].tolist(),
            }
        with open(os.path.join(HERE, f"ref_{name}.json"), "w") as f:
            json.dump(res, f, indent=1)
    finally:
        shutil.rmtree(tmp)


def main():
    O.build(ref=True)
    which = sys.argv[1] if len(sys.argv) > 1 else "all"
    if which == "all":
        breakpoints()
        kat_primitives()
        for c in CONFIGS:
            ref_config(*c)
    if which in ("all", "config1"):
        ref_config1(*CONFIG1)


if __name__ == "__main__":
    main()
