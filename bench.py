#!/usr/bin/env python
"""bench.py -- exact k-NN queries/s on one B200 at 25M x 256 (Hercules path).

Collection: 25,000,000 z-normalised random walks of length 256 (25.6 GB
float32 resident in HBM; seeded synthetic data, dataset seed 1184), leaf
size 100,000, built into the Hercules EAPCA index on the GPU.

Headline workload (a step): one batch of 4,096 queries answered exactly by
the batched path (hg_knn_batch_device): equal thirds of noisy queries (a
random dataset series plus N(0, sigma^2) noise, sigma^2 = 0.01 / 0.1 / 1.0,
z-normalised) plus 10% fresh random walks, k in {1, 10, 100} (every
(sigma^2, k) pair in equal shares).  `value` is queries per second over the
timed steps (CUDA events on the stream, the collection and the step's
queries already in HBM); `e2e` is the same through hg_knn_batch with the
queries in pinned host memory and the answers copied back every step.

Beside it, on the same collection:
  plain      the plain per-query path (hg_knn_device) on 1,000 noisy queries
             (sigma^2 in thirds), k = 1 and k = 10, with the leaf-scan
             kernel's HBM roofline (`leaf_scan`);
  pscan      the unindexed full scan (HG_MODE_PSCAN), its answers checked
             against the plain path's, with the reference's multi-threaded
             CPU PSCAN on a bounded sample;
  fp64_oracle  answers of a timed batch and of both plain legs against an
             FP64 brute force over the whole collection;
  parity     the reference's own exact search (oracle/_ref/hercules, built
             from the reference sources) over the index files the GPU
             wrote, on a sample of timed queries: its printed distances and
             answer-leaf positions against the GPU's;
  index      SHA-256 digests of the index files the GPU wrote (the
             `--impl reference` arm prints the same digests for the files
             the oracle's restatement of the reference build writes).

The BF16 copy of the collection (12.8 GB) and the raw rows (25.6 GB) are far
larger than L2 (126 MB); every step streams them from HBM, so no L2 flush is
needed between steps.

--impl reference times the reference Hercules query path
(oracle/_ref/hercules, compiled from the reference's own sources, all host
cores) on queries drawn from the same batches.  That process loads nothing
of hercules_b200: the collection and the queries come from the oracle's
restatement of the generator, and the index files from the oracle's
restatement of the reference's one-worker build.

Multi-GPU (torchrun, N > 1): by default the collection is split into N
row-range shards, each rank builds and searches its own, and every batch's
per-shard answers are all-gathered over NCCL and merged on the device inside
the timed region (strong scaling: the total work is fixed).  --multi replica
gives every rank a full copy and its own queries instead (weak scaling, no
data-path collective).
"""
import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "exact k-NN queries/s @25Mx256, batched-BF16 vs plain GPU; leaf-scan HBM GB/s"
UNIT = "queries/s"
DATA_SEED = 1184
QUERY_SEED = 14784
FRESH_SEED = 99991
K_CYCLE = (1, 10, 100)


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=25_000_000)
    p.add_argument("--L", type=int, default=256)
    p.add_argument("--leaf", type=int, default=100_000)
    p.add_argument("--batch", type=int, default=4096, help="queries per batched step")
    p.add_argument("--fresh-frac", type=float, default=0.1)
    p.add_argument("--plain-queries", type=int, default=1000, help="queries through the plain path")
    p.add_argument("--plain-ks", default="1,10", help="k of the plain legs (the last one carries the roofline)")
    p.add_argument("--data", choices=["walks", "unit"], default="walks",
                   help="z-normalised random walks, or unit-normalised Gaussian vectors")
    p.add_argument("--sigma2", default="0.01,0.1,1.0", help="noise levels of the noisy queries, in equal shares")
    p.add_argument("--ks", default="1,10,100", help="k of the batched queries, cycling")
    p.add_argument("--cpu-sample-queries", type=int, default=6,
                   help="timed queries answered by the reference's serial exact search (baseline + parity)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-queries-per-step", type=int, default=2)
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch parameters")
    p.add_argument("--multi", choices=["shard", "replica"], default="shard",
                   help="N > 1: row-range shards of one collection (all-gather + merge per batch) or full replicas")
    return p.parse_args()


SIGMA2 = (0.01, 0.1, 1.0)


def sigma2_for(nq, offset=0, levels=SIGMA2):
    cyc = np.array(levels, dtype=np.float64)
    return cyc[(np.arange(nq) + offset) % len(cyc)]


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                                       "--format=csv,noheader,nounits", "-lms", "50"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args, backend=None):
    """One process per GPU (torchrun environment); replicas exchange only the
    step times (max over ranks)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        if backend is None:
            backend = "gloo" if args.impl == "reference" else "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return rank, world, local


def rank_offset(rank):
    """Query-seed offset of a replica: every rank answers its own queries."""
    return rank * 7919


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peaks_all():
    """Roofline denominators: the driver-measured copy bandwidth and bf16
    GEMM throughput of this pool's B200s, else the earlier pool figures."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm": float(d["hbm_gbs"]), "bf16": float(d["bf16_tflops"]),
                "bf16_sustained": float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "source": "measured"}
    return {"hbm": 6650.0, "bf16": 1590.0, "bf16_sustained": 1400.0, "source": "fallback"}


def profile_json(name):
    """A committed ncu summary figure (profiles/<name>), or None."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p))
    except ValueError:
        return None


def build_collection(args, torch, H, device):
    n, L = args.n, args.L
    X = torch.empty((n, L), dtype=torch.float32, device=device)
    if args.data == "unit":
        H.generate_unit_vectors_device(DATA_SEED, n, L, X.data_ptr(), device=device)
    else:
        H.generate_walks_device(DATA_SEED, n, L, X.data_ptr(), device=device)
    torch.cuda.synchronize()
    return X


def make_queries(args, torch, H, X, nq, device, offset):
    Q = torch.empty((nq, args.L), dtype=torch.float32, device=device)
    gen = H.generate_unit_queries_device if args.data == "unit" else H.generate_queries_device
    gen(QUERY_SEED + offset, X.data_ptr(), args.n, args.L, sigma2_for(nq, levels=levels_of(args)), Q.data_ptr(),
        device=device)
    torch.cuda.synchronize()
    return Q


def levels_of(args):
    return tuple(float(x) for x in args.sigma2.split(","))


def ks_of(args):
    return tuple(int(x) for x in args.ks.split(","))


def batch_ks(args):
    """k of each query of a batch: the noise level cycles with the query
    index and k with the index divided by the number of levels, so every
    (sigma^2, k) pair has an equal share."""
    kc = np.array(ks_of(args), np.uint32)
    return kc[(np.arange(args.batch) // len(levels_of(args))) % len(kc)]


def fresh_count(args):
    return int(round(args.batch * args.fresh_frac))


def make_batches(args, torch, H, X, nbatches, device, offset):
    """nbatches batches of args.batch queries: noisy queries (sigma^2 in
    equal shares) followed by fresh random walks (args.fresh_frac)."""
    nb = args.batch
    nf = fresh_count(args)
    Q = torch.empty((nbatches, nb, args.L), dtype=torch.float32, device=device)
    gen = H.generate_unit_queries_device if args.data == "unit" else H.generate_queries_device
    fresh = H.generate_unit_vectors_device if args.data == "unit" else H.generate_walks_device
    for i in range(nbatches):
        gen(QUERY_SEED + offset + i, X.data_ptr(), args.n, args.L, sigma2_for(nb - nf, levels=levels_of(args)),
            Q[i].data_ptr(), device=device)
        if nf:
            fresh(FRESH_SEED + offset, nf, args.L, Q[i, nb - nf:].data_ptr(), first=(offset + i) * nf, device=device)
    torch.cuda.synchronize()
    return Q, batch_ks(args)


def batch_on_host(args, O, i, offset=0):
    """Batch i of make_batches computed on the host by the oracle's
    restatement of the generator (the same bits), for the CPU-only arm."""
    nb = args.batch
    nf = fresh_count(args)
    unit = args.data == "unit"
    noisy, _ = O.gen_queries(DATA_SEED, QUERY_SEED + offset + i, args.n, args.L,
                             sigma2_for(nb - nf, levels=levels_of(args)), unit=unit)
    parts = [noisy]
    if nf:
        parts.append(O.gen_rows(FRESH_SEED + offset, nf, args.L, first=(offset + i) * nf, unit=unit))
    return np.ascontiguousarray(np.concatenate(parts, 0)), batch_ks(args)


def config_of(args):
    """The workload, identical in both arms' JSON lines."""
    what = "z-normalised random walks" if args.data == "walks" else "unit-normalised Gaussian vectors"
    return {"workload": "batched exact k-NN, %d x %d float32 %s, leaf %d, %d queries/step, k in {%s}, "
                        "sigma2 in equal shares %s + %d%% fresh %s"
                        % (args.n, args.L, what, args.leaf, args.batch, ",".join(map(str, ks_of(args))),
                           "/".join(map(str, levels_of(args))), int(round(100 * args.fresh_frac)),
                           "walks" if args.data == "walks" else "vectors"),
            "n": args.n, "L": args.L, "leaf_size": args.leaf, "queries_per_step": args.batch,
            "k": list(ks_of(args)), "data": args.data,
            "l2": "inputs (%.1f GB f32 + %.1f GB bf16) larger than L2; no flush needed"
                  % (args.n * args.L * 4 / 1e9, args.n * args.L * 2 / 1e9),
            "parallelism": parallelism_of(args)}


def parallelism_of(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world == 1:
        return "single GPU"
    if args.multi == "replica":
        return "replica per GPU (each rank its own queries)"
    return "%d row-range shards; every rank answers the whole batch, NCCL all-gather of the k nearest + merge" % world


def fp64_oracle_check(args, torch, H, groups, device):
    """FP64 brute force over the whole collection (regenerated chunk by chunk
    from the same seed) for groups of answered queries, each
    (name, Q [s, L] device, ks [s], D [s, >=kmax], I [s, >=kmax]): recall of
    the returned ids against the FP64 k nearest, and the relative error of
    the returned FP32 distances against the FP64 distances of the same rows.
    One pass over the collection serves every group."""
    n, L = args.n, args.L
    names, qs, kss, ours_i, ours_d = [], [], [], [], []
    width = max(int(np.max(ks)) for _, _, ks, _, _ in groups)
    for name, Q, ks, D, I in groups:
        s = Q.shape[0]
        kq = np.broadcast_to(np.asarray(ks, np.int64), (s,))
        kmax = int(kq.max())
        names.append((name, s))
        qs.append(Q.double())
        kss.append(kq)
        pad_i = torch.full((s, width), -1, dtype=torch.int64, device=device)
        pad_d = torch.full((s, width), float("nan"), dtype=torch.float64, device=device)
        pad_i[:, :kmax] = I[:, :kmax]
        pad_d[:, :kmax] = D[:, :kmax].double()
        ours_i.append(pad_i)
        ours_d.append(pad_d)
    q = torch.cat(qs, 0)
    ks_all = np.concatenate(kss)
    ours = torch.cat(ours_i, 0)
    ours_dd = torch.cat(ours_d, 0)
    s = q.shape[0]
    kmax = int(ks_all.max())
    gen = H.generate_unit_vectors_device if args.data == "unit" else H.generate_walks_device
    chunk = max(1, min(n, (1 << 28) // L))
    buf = torch.empty((chunk, L), dtype=torch.float32, device=device)
    best_d = torch.full((s, kmax), float("inf"), dtype=torch.float64, device=device)
    best_i = torch.full((s, kmax), -1, dtype=torch.int64, device=device)
    d64_ours = torch.full((s, width), float("nan"), dtype=torch.float64, device=device)
    qn = (q * q).sum(1)
    for first in range(0, n, chunk):
        m = min(chunk, n - first)
        gen(DATA_SEED, m, L, buf.data_ptr(), first=first, device=device)
        x = buf[:m].double()
        d = (qn[:, None] + (x * x).sum(1)[None, :] - 2.0 * (q @ x.T)).clamp_min_(0.0)
        ids = torch.arange(first, first + m, device=device)
        cd = torch.cat([best_d, d], 1)
        ci = torch.cat([best_i, ids[None, :].expand(s, m)], 1)
        best_d, pos = torch.topk(cd, kmax, dim=1, largest=False, sorted=True)
        best_i = torch.gather(ci, 1, pos)
        inside = (ours >= first) & (ours < first + m)
        if inside.any():
            rr, cc = inside.nonzero(as_tuple=True)
            d64_ours[rr, cc] = d[rr, ours[rr, cc] - first]
    torch.cuda.synchronize()
    out = {"how": "FP64 brute force over all %d rows, regenerated from the data seed in chunks" % n}
    row = 0
    for name, cnt in names:
        hits, total, max_rel = 0, 0, 0.0
        for j in range(row, row + cnt):
            k = int(ks_all[j])
            a = set(ours[j, :k].tolist())
            b = set(best_i[j, :k].tolist())
            hits += len(a & b)
            total += k
            d64 = d64_ours[j, :k]
            rel = ((ours_dd[j, :k] - d64).abs() / d64.clamp_min(1e-30)).max()
            max_rel = max(max_rel, float(rel))
        out[name] = {"queries": cnt, "pairs": total, "recall_vs_fp64_topk": round(hits / max(total, 1), 6),
                     "max_rel_err_vs_fp64": max_rel}
        row += cnt
    return out


_TSV_ANSWER = ("Query_exact_distance", "Query_exact_node_file_pos")


def cpu_reference_run(args, index_dir, queries_host, threads, extra=(), k=10):
    """Runs the reference CLI over the written index.  Returns per-query
    seconds from its own Query_total_time_secs lines, the wall time, and its
    printed answers {query number: {"dist": [...], "pos": [...]}} (the %f
    square-root distances and answer-leaf file positions, by rank)."""
    from oracle import oracle as O
    binary = O.REF_BIN
    qfile = os.path.join(index_dir, "bench_queries.bin")
    np.ascontiguousarray(queries_host, np.float32).tofile(qfile)
    nq = queries_host.shape[0]
    cmd = [binary, "--mode", "1", "--serial", "1", "--num-threads", str(threads), "--k", str(k),
           "--queries", qfile, "--queries-size", str(nq), "--index-path", index_dir, *extra]
    t0 = time.perf_counter()
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=1800, cwd=index_dir)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        raise RuntimeError("reference query failed: " + r.stderr[-500:])
    per_q, ans = {}, {}
    for line in r.stdout.splitlines():
        parts = line.split("\t")
        if len(parts) != 5:
            continue
        if parts[0] == "Query_total_time_secs":
            per_q.setdefault(int(parts[3]), 0.0)
            per_q[int(parts[3])] += float(parts[1])
        elif parts[0] in _TSV_ANSWER:
            a = ans.setdefault(int(parts[3]), {"dist": {}, "pos": {}})
            a["dist" if parts[0] == _TSV_ANSWER[0] else "pos"][int(parts[4])] = parts[1]
    answers = {qn: {"dist": [a["dist"][r] for r in sorted(a["dist"])], "pos": [a["pos"][r] for r in sorted(a["pos"])]}
               for qn, a in ans.items()}
    return per_q, wall, answers


def file_digest(path, chunk=1 << 26):
    """SHA-256 of the concatenated SHA-256 digests of the file's 64 MiB
    chunks, hashed on every host core."""
    import hashlib
    from concurrent.futures import ThreadPoolExecutor
    size = os.path.getsize(path)

    def one(off):
        with open(path, "rb") as f:
            f.seek(off)
            return hashlib.sha256(f.read(chunk)).digest()

    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        parts = list(ex.map(one, range(0, max(size, 1), chunk)))
    return hashlib.sha256(b"".join(parts)).hexdigest()


def index_digests(d):
    return {f: file_digest(os.path.join(d, f)) for f in ("root.idx", "leaves_raw.idx", "leaves_sims.idx")}


def cpu_pscan_leg(args, H, queries_host, k):
    """The reference's PSCAN (oracle/_ref/pscan, built from code/pscan) with
    every host core on a bounded sample: the queries over the first m rows
    of the same collection (about 1 GB, regenerated on the host with the
    same seed), its Query_total_time_secs scaled by n / m to the full size."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    if not os.path.exists(O.REF_PSCAN):
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": "unavailable: oracle/_ref/pscan not built"}
    m = int(min(args.n, max(1, (1 << 28) // args.L)))
    d = None
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(base)
            if st.f_bavail * st.f_frsize > m * args.L * 4 * 1.5:
                d = tempfile.mkdtemp(prefix="hg_bench_pscan_", dir=base)
                break
        except OSError:
            continue
    if d is None:
        return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": "unavailable: no host space for the sample"}
    try:
        gen = H.generate_unit_vectors if args.data == "unit" else H.generate_walks
        data = os.path.join(d, "data.bin")
        gen(DATA_SEED, m, args.L).tofile(data)
        qfile = os.path.join(d, "queries.bin")
        np.ascontiguousarray(queries_host, np.float32).tofile(qfile)
        nq = queries_host.shape[0]
        cmd = [O.REF_PSCAN, "--dataset", data, "--queries", qfile, "--dataset-size", str(m),
               "--queries-size", str(nq), "--timeseries-size", str(args.L), "--k", str(k),
               "--num-query-threads", str(cores + 1), "--dbsize", "120000"]
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900, cwd=d)
        if r.returncode != 0:
            return {"value": None, "unit": UNIT, "cores": cores, "kind": "reference",
                    "sample": "unavailable: reference PSCAN failed: " + r.stderr[-200:]}
        secs = 0.0
        for line in r.stdout.splitlines():
            parts = line.split("\t")
            if len(parts) == 5 and parts[0] == "Query_total_time_secs":
                secs += float(parts[1])
        per_q = secs / nq * (args.n / m)
        return {"value": round(1.0 / per_q, 4) if per_q > 0 else None, "unit": UNIT, "cores": cores,
                "kind": "reference",
                "sample": "%d queries (k = %d) over the first %d rows of the collection; Query_total_time_secs "
                          "scaled by %d / %d" % (nq, k, m, args.n, m)}
    finally:
        shutil.rmtree(d, ignore_errors=True)


def write_index_for_cpu(ix, args):
    """The index in the reference's format where the host can read it fast."""
    d = host_index_dir(args.n * args.L * 4 * 1.3, "hg_bench_idx_")
    if d is not None:
        ix.write(d, buffer_mb=64.0)
    return d


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, rank, world, local)
    if world > 1 and args.multi == "shard":
        return run_sharded(args, rank, world, local)
    import torch
    import hercules_b200 as H
    from hercules_b200 import build as B
    B.build()
    torch.cuda.set_device(local)
    device = local
    steps, warm, nb = args.steps, args.warmup, args.batch
    t_setup = time.perf_counter()
    X = build_collection(args, torch, H, device)
    off = rank_offset(rank)
    Qb, ks = make_batches(args, torch, H, X, steps + warm, device, offset=off)
    Qe, _ = make_batches(args, torch, H, X, steps + warm, device, offset=off + 5000)
    Qp = make_queries(args, torch, H, X, args.plain_queries, device, offset=off + 9000)
    t0 = time.perf_counter()
    ix = H.HerculesIndex.build_device(X.data_ptr(), args.n, args.L, args.leaf, device=device)
    build_s = time.perf_counter() - t0
    del X
    torch.cuda.empty_cache()
    kmax = int(ks.max())
    D = torch.empty((nb, kmax), dtype=torch.float32, device=device)
    I = torch.empty((nb, kmax), dtype=torch.int64, device=device)
    stream = torch.cuda.current_stream().cuda_stream

    def batch_step(i):
        return ix.knn_batch_device(Qb[i].data_ptr(), nb, ks, kmax, D.data_ptr(), I.data_ptr(), stream=stream)

    t1 = time.perf_counter()
    batch_step(0)  # the first call also builds the BF16 copy of the collection
    torch.cuda.synchronize()
    prep_s = time.perf_counter() - t1
    # launch parameters tuned on a warm-up batch, before the timed region
    tuning = ix.tuning() if args.no_autotune else ix.autotune_device(Qb[0].data_ptr(), nb, ks, kmax, stream=stream)
    for i in range(1, warm):
        batch_step(i)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    agg = {}
    for i in range(warm, warm + steps):
        st = batch_step(i)
        for kk, v in st.items():
            agg[kk] = agg.get(kk, 0) + v
        agg["err_max_max"] = max(agg.get("err_max_max", 0.0), st["err_max"])
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, device=torch.device("cuda", device))
    total_q = nb * steps * world
    value = total_q / (ms / 1000.0)
    last = warm + steps - 1  # D / I hold the answers of this batch

    # end to end through the host API: pinned host queries in, answers out
    Qh = torch.empty(tuple(Qe.shape), dtype=torch.float32, pin_memory=True)
    Qh.copy_(Qe.cpu())
    Qhn = Qh.numpy()
    for i in range(warm):
        ix.knn_batch(Qhn[i], ks)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(warm, warm + steps):
        ix.knn_batch(Qhn[i], ks)
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, device=torch.device("cuda", device))
    e2e_value = total_q / e2e_s

    # the plain per-query path on 1,000 noisy queries, one leg per k; the
    # last leg times every scan launch (roofline of the leaf scan)
    plain_ks = [int(x) for x in args.plain_ks.split(",")]
    npl = args.plain_queries
    plain, plain_ans = {}, {}
    for j, pk in enumerate(plain_ks):
        Dp = torch.empty((npl, pk), dtype=torch.float32, device=device)
        Ip = torch.empty((npl, pk), dtype=torch.int64, device=device)
        ix.knn_device(Qp.data_ptr(), min(8, npl), pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream, use_lb_sax=True)
        torch.cuda.synchronize()
        p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        prof = j == len(plain_ks) - 1
        p0.record()
        pst = ix.knn_device(Qp.data_ptr(), npl, pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream, use_lb_sax=True,
                            profile=prof)
        p1.record()
        torch.cuda.synchronize()
        qps = npl / (p0.elapsed_time(p1) / 1000.0)
        plain["k%d" % pk] = {"value": round(qps, 2), "unit": UNIT, "queries": npl, "k": pk,
                             "profiled": prof, "leaves_scanned_per_query": pst["leaves_scanned"] / npl,
                             "rows_visited_per_query": pst["rows_visited"] / npl}
        plain_ans[pk] = (Dp, Ip)
        if prof:
            plain_st = pst
    pk = plain_ks[-1]
    plain_qps = plain["k%d" % pk]["value"]

    # PSCAN (every row of the collection per query, HG_MODE_PSCAN): the
    # unindexed baseline, HBM-bound; its answers must equal the plain path's
    npq = max(1, min(4, npl))
    Ds = torch.empty((npq, pk), dtype=torch.float32, device=device)
    Is = torch.empty((npq, pk), dtype=torch.int64, device=device)
    ix.knn_device(Qp.data_ptr(), 1, pk, Ds.data_ptr(), Is.data_ptr(), stream=stream, mode=H.MODE_PSCAN)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    sst = ix.knn_device(Qp.data_ptr(), npq, pk, Ds.data_ptr(), Is.data_ptr(), stream=stream, mode=H.MODE_PSCAN,
                        profile=True)
    s1.record()
    torch.cuda.synchronize()
    pscan_ms = s0.elapsed_time(s1)
    pscan_bytes = 32.0 * sst["chunks_loaded"] + 8.0 * sst["rows_completed"]
    pscan_scan_s = (sst["scan_ms"] if sst["scan_ms"] > 0 else pscan_ms) / 1000.0
    pscan_gbs = pscan_bytes / pscan_scan_s / 1e9
    Dpk, Ipk = plain_ans[pk]
    pscan_same = bool(torch.equal(Ds.view(torch.int32), Dpk[:npq].contiguous().view(torch.int32))
                      and torch.equal(Is, Ipk[:npq]))
    pscan = {"value": round(npq / (pscan_ms / 1000.0), 2), "unit": UNIT, "queries": npq, "k": pk,
             "path": "hg_knn_device, HG_MODE_PSCAN (every row, early abandon at the running k-th distance)",
             "answers_equal_plain_path": pscan_same,
             "scan": {"kernel": "k_ed_stream", "achieved": round(pscan_gbs, 1), "unit": "GB/s",
                      "frac": round(pscan_gbs / measured_peaks_all()["hbm"], 4),
                      "algorithmic_bytes_per_query": pscan_bytes / npq}}

    # answers of the last timed batch and of both plain legs against FP64
    ns = min(32, nb)
    groups = [("batched", Qb[last, :ns], ks[:ns], D[:ns], I[:ns])]
    npk = min(32, npl)
    for pk_, (Dp, Ip) in plain_ans.items():
        groups.append(("plain_k%d" % pk_, Qp[:npk], np.full(npk, pk_), Dp[:npk], Ip[:npk]))
    fp64 = fp64_oracle_check(args, torch, H, groups, device)

    cpu_baseline, parity, index = None, None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sample = sample_positions(args, args.cpu_sample_queries)
        cpu_q = Qb[last, sample].cpu().numpy()
        cpu_k = ks[sample]
        cpu_d = D[sample].cpu().numpy()
        cpu_i = I[sample].cpu().numpy()
        cpu_baseline, parity, index = cpu_baseline_leg(args, ix, cpu_q, cpu_k, cpu_d, cpu_i)
        pscan["cpu_baseline"] = cpu_pscan_leg(args, H, Qp[:npq].cpu().numpy(), pk)
    ix.close()

    # roofline of the dominant kernel, the tensor-core filter k_umma_filter:
    # algorithmic FLOPs = 2 L per (query, row) pair it evaluated, over its
    # summed launch time (%globaltimer stamps around every filter phase)
    peaks = measured_peaks_all()
    gemm_s = agg["gemm_ms"] / 1000.0
    flops = 2.0 * args.L * agg["bf16_pairs"]
    achieved_tf = flops / gemm_s / 1e12 if gemm_s > 0 else 0.0
    tr = profile_json("k_umma_filter_traffic.json")
    traffic = None
    if tr and tr.get("dram_bytes_per_row_pass"):
        traffic = tr["dram_bytes_per_row_pass"] * args.n
    roofline = {"bound": "tensor", "kernel": "k_umma_filter", "achieved": round(achieved_tf, 1),
                "peak": peaks["bf16_sustained"], "unit": "TFLOP/s",
                "frac": round(achieved_tf / peaks["bf16_sustained"], 4),
                "peak_source": peaks["source"] + " sustained bf16 (the filter runs inside seconds-long steps)",
                "traffic": traffic, "algorithmic_flops_per_step": flops / steps,
                "avg_ms_per_step": agg["gemm_ms"] / steps, "pairs_per_step": agg["bf16_pairs"] / steps}
    # leaf scan of the plain path: k_ed_stream's algorithmic bytes = 32 B per
    # 8-float chunk computed + 4 B list entry per row started + 8 B id per
    # finished row, over its summed launch time
    pst = plain_st
    launches = int(pst["scan_launches"])
    alg_bytes = 32.0 * pst["chunks_loaded"] + 4.0 * pst["rows_visited"] + 8.0 * pst["rows_completed"]
    scan_s = pst["scan_ms"] / 1000.0
    ed_gbs = alg_bytes / scan_s / 1e9 if scan_s > 0 else 0.0
    tre = profile_json("k_ed_stream_traffic.json")
    ed_traffic = None
    if tre and tre.get("dram_bytes_per_algorithmic_byte"):
        ed_traffic = tre["dram_bytes_per_algorithmic_byte"] * alg_bytes / max(launches, 1)
    leaf_scan = {"bound": "hbm", "kernel": "k_ed_stream", "achieved": round(ed_gbs, 1), "peak": peaks["hbm"],
                 "unit": "GB/s", "frac": round(ed_gbs / peaks["hbm"], 4), "peak_source": peaks["source"],
                 "traffic": ed_traffic, "algorithmic_bytes_per_launch": alg_bytes / max(launches, 1),
                 "avg_launch_ms": pst["scan_ms"] / max(launches, 1), "launches": launches}
    # the LB_SAX filter of the plain path: 16 B word per row considered + 4 B
    # per survivor written, over its summed launch time
    flt_s = pst["filter_ms"] / 1000.0
    flt_bytes = 16.0 * pst["rows_considered"] + 4.0 * (pst["rows_considered"] - pst["rows_lbsax_pruned"])
    flt_gbs = flt_bytes / flt_s / 1e9 if flt_s > 0 else 0.0
    lbsax = {"bound": "hbm", "kernel": "k_lbsax_filter", "achieved": round(flt_gbs, 1), "peak": peaks["hbm"],
             "unit": "GB/s", "frac": round(flt_gbs / peaks["hbm"], 4),
             "launches": int(pst["filter_launches"]),
             "avg_launch_ms": pst["filter_ms"] / max(int(pst["filter_launches"]), 1),
             "share_of_plain_device_time": round(pst["filter_ms"] / max(pst["device_ms"], 1e-9), 4)}
    # the exact re-rank of the batched path: 32 B per chunk it computed + 4 B
    # per survivor row it read from the buckets, over its phase time (plan,
    # segments and merge, %globaltimer stamps)
    rr_bytes = 32.0 * agg["chunks_loaded"] + 4.0 * agg["rows_visited"]
    rr_s = agg["rerank_ms"] / 1000.0
    rr_gbs = rr_bytes / rr_s / 1e9 if rr_s > 0 else 0.0
    rerank = {"bound": "hbm", "kernels": "k_rerank_plan + k_rerank_part + k_rerank_merge",
              "achieved": round(rr_gbs, 1), "peak": peaks["hbm"], "unit": "GB/s",
              "frac": round(rr_gbs / peaks["hbm"], 4), "bytes_per_step": rr_bytes / steps,
              "ms_per_step": agg["rerank_ms"] / steps}
    plain.update({"value": plain_qps, "unit": UNIT, "k": pk,
                  "batched_over_plain": round(value / plain_qps, 2) if plain_qps > 0 else None,
                  "path": "hg_knn_device (one query at a time, LB_SAX on); value = the k = %d leg" % pk})
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 filter (fp32 accumulate) + f32 exact re-rank",
        "data": "synthetic (seeded z-normalised random walks; noisy and fresh queries)",
        "config": config_of(args),
        "tuning": dict({k: tuning[k] for k in ("filter_cta_pair", "filter_tiles_per_item", "bound_tiles_per_item",
                                                "rerank_blocks_per_sm", "approx_blocks_per_sm")},
                       tuned=not args.no_autotune),
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": nb * args.L * 4,
                "d2h_bytes_per_step": nb * kmax * (4 + 8)},
        "gpu_launches": int(agg["kernel_launches"]),
        "roofline": roofline,
        "leaf_scan": leaf_scan,
        "lbsax_filter": lbsax,
        "rerank": rerank,
        "plain": plain,
        "cpu_baseline": cpu_baseline,
        "parity": parity,
        "index": index,
        "pscan": pscan,
        "clocks": ck,
        "certified_bound": {"err_mean": agg["err_mean"] / steps, "err_max": agg["err_max_max"],
                            "err_over_bound_mean": agg["err_over_bound"] / steps,
                            "what": "err(q, work item) of the filter pass over every row: "
                                    "d~ - err <= B_q keeps every row within B_q"},
        "fp64_oracle": fp64,
        "stats": {"survivors_per_query": agg["survivors"] / (nb * steps),
                  "survivor_fraction": agg["survivors"] / max(agg["bf16_pairs"], 1),
                  "leaf_pairs_kept_fraction": (agg["leaf_pairs_kept"] / agg["leaf_pairs"]) if agg["leaf_pairs"] else None,
                  "filter_pairs_fraction": agg["bf16_pairs"] / (float(args.n) * nb * steps),
                  "rerank_rows_per_query": agg["rows_visited"] / (nb * steps),
                  "retried_queries_per_step": agg["retried_queries"] / steps,
                  "fallback_queries_per_step": agg["fallback_queries"] / steps,
                  "bound_ms_per_step": agg["bound_ms"] / steps, "filter_ms_per_step": agg["gemm_ms"] / steps,
                  "rerank_ms_per_step": agg["rerank_ms"] / steps, "fallback_ms_per_step": agg["fallback_ms"] / steps,
                  "first_call_prep_s": round(prep_s, 2), "index_build_s": round(build_s, 2),
                  "setup_s": round(time.perf_counter() - t_setup, 2)},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def make_batches_seeded(args, torch, H, nbatches, device, offset):
    """make_batches without the collection on the device: each noisy query's
    base row is regenerated from the data seed (the same bits)."""
    nb = args.batch
    nf = fresh_count(args)
    unit = args.data == "unit"
    Q = torch.empty((nbatches, nb, args.L), dtype=torch.float32, device=device)
    fresh = H.generate_unit_vectors_device if unit else H.generate_walks_device
    for i in range(nbatches):
        H.generate_queries_seeded_device(DATA_SEED, QUERY_SEED + offset + i, args.n, args.L,
                                         sigma2_for(nb - nf, levels=levels_of(args)), Q[i].data_ptr(), unit=unit,
                                         device=device)
        if nf:
            fresh(FRESH_SEED + offset, nf, args.L, Q[i, nb - nf:].data_ptr(), first=(offset + i) * nf, device=device)
    torch.cuda.synchronize()
    return Q, batch_ks(args)


def run_sharded(args, rank, world, local):
    """N > 1: rank r holds rows shard_range(n, N, r) of the collection as its
    own index and answers every query of each batch on it; one NCCL
    all-gather of the k (distance, id) pairs per query and a merge on the
    device give the answers of the whole collection (hercules_b200.shard).
    The timed region holds the batched search, the collective and the merge;
    the total work is fixed as N grows (strong scaling)."""
    import torch
    import hercules_b200 as H
    from hercules_b200 import build as B
    from hercules_b200.shard import shard_range, sharded_batch_answers
    B.build()
    torch.cuda.set_device(local)
    device = local
    dev = torch.device("cuda", device)
    steps, warm, nb = args.steps, args.warmup, args.batch
    t_setup = time.perf_counter()
    first, count = shard_range(args.n, world, rank)
    X = torch.empty((count, args.L), dtype=torch.float32, device=device)
    gen = H.generate_unit_vectors_device if args.data == "unit" else H.generate_walks_device
    gen(DATA_SEED, count, args.L, X.data_ptr(), first=first, device=device)
    torch.cuda.synchronize()
    ix = H.HerculesIndex.build_device(X.data_ptr(), count, args.L, args.leaf, device=device)
    del X
    torch.cuda.empty_cache()
    Qb, ks = make_batches_seeded(args, torch, H, steps + warm, device, offset=0)
    kmax = int(ks.max())
    D = torch.empty((nb, kmax), dtype=torch.float32, device=device)
    I = torch.empty((nb, kmax), dtype=torch.int64, device=device)
    stream = torch.cuda.current_stream().cuda_stream

    def step(qptr):
        st = ix.knn_batch_device(qptr, nb, ks, kmax, D.data_ptr(), I.data_ptr(), stream=stream)
        md, mi = sharded_batch_answers(D, I, first, ks, kmax)
        return st, md, mi

    step(Qb[0].data_ptr())  # the first call also builds the BF16 copy of the shard
    torch.cuda.synchronize()
    tuning = ix.tuning() if args.no_autotune else ix.autotune_device(Qb[0].data_ptr(), nb, ks, kmax, stream=stream)
    for i in range(1, warm):
        step(Qb[i].data_ptr())
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    agg = {}
    for i in range(warm, warm + steps):
        st, md, mi = step(Qb[i].data_ptr())
        for kk, v in st.items():
            agg[kk] = agg.get(kk, 0) + v
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = max_over_ranks(e0.elapsed_time(e1), world, device=dev)
    value = nb * steps / (ms / 1000.0)
    last_d, last_i = md, mi

    # end to end: pinned host queries in, merged answers back to pinned host
    # memory, every step
    Qe, _ = make_batches_seeded(args, torch, H, steps + warm, device, offset=5000)
    Qh = torch.empty(tuple(Qe.shape), dtype=torch.float32, pin_memory=True)
    Qh.copy_(Qe.cpu())
    del Qe
    Qd = torch.empty((nb, args.L), dtype=torch.float32, device=device)
    Dh = torch.empty((nb, kmax), dtype=torch.float32, pin_memory=True)
    Ih = torch.empty((nb, kmax), dtype=torch.int64, pin_memory=True)

    def e2e_step(i):
        Qd.copy_(Qh[i], non_blocking=True)
        _, md2, mi2 = step(Qd.data_ptr())
        Dh.copy_(md2, non_blocking=True)
        Ih.copy_(mi2, non_blocking=True)
        torch.cuda.synchronize()

    for i in range(warm):
        e2e_step(i)
    barrier(world)
    t0 = time.perf_counter()
    for i in range(warm, warm + steps):
        e2e_step(i)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, device=dev)
    e2e_value = nb * steps / e2e_s

    fp64 = None
    if rank == 0:
        ns = 32
        fp64 = fp64_oracle_check(args, torch, H, [("sharded_batched", Qb[warm + steps - 1, :ns], ks[:ns],
                                                   last_d[:ns], last_i[:ns])], device)
    barrier(world)
    ix.close()
    peaks = measured_peaks_all()
    gemm_s = agg["gemm_ms"] / 1000.0
    flops = 2.0 * args.L * agg["bf16_pairs"]
    achieved_tf = flops / gemm_s / 1e12 if gemm_s > 0 else 0.0
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "bf16 filter (fp32 accumulate) + f32 exact re-rank",
        "data": "synthetic (seeded z-normalised random walks; noisy and fresh queries)",
        "config": config_of(args),
        "tuning": dict({k: tuning[k] for k in ("filter_cta_pair", "filter_tiles_per_item", "bound_tiles_per_item",
                                                "rerank_blocks_per_sm", "approx_blocks_per_sm")},
                       tuned=not args.no_autotune),
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": nb * args.L * 4,
                "d2h_bytes_per_step": nb * kmax * (4 + 8)},
        "gpu_launches": int(agg["kernel_launches"]),
        "roofline": {"bound": "tensor", "kernel": "k_umma_filter (rank 0's shard)", "achieved": round(achieved_tf, 1),
                     "peak": peaks["bf16_sustained"], "unit": "TFLOP/s",
                     "frac": round(achieved_tf / peaks["bf16_sustained"], 4),
                     "peak_source": peaks["source"] + " sustained bf16", "traffic": None},
        "shard": {"rows_rank0": count, "collective": "torch.distributed all_gather (NCCL) of [batch, kmax] "
                                                     "distances and ids, merge_topk_torch on the device"},
        "clocks": ck,
        "fp64_oracle": fp64,
        "stats": {"filter_ms_per_step_rank0": agg["gemm_ms"] / steps,
                  "rerank_ms_per_step_rank0": agg["rerank_ms"] / steps,
                  "bound_ms_per_step_rank0": agg["bound_ms"] / steps,
                  "setup_s": round(time.perf_counter() - t_setup, 2)},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    import torch.distributed as dist
    dist.destroy_process_group()


def sample_positions(args, m):
    """m query positions of a batch spread over it: every k and every noise
    level appears (k cycling with the sample index, the level shifted by one
    per round of k), the last one a fresh walk when the batch has some."""
    nb, nlev, nk = args.batch, len(levels_of(args)), len(ks_of(args))
    nf = fresh_count(args)
    out = []
    for t in range(m):
        want_k = t % nk
        fresh = nf > 0 and t == m - 1
        lo, hi = (nb - nf, nb) if fresh else (t * (nb - nf) // max(m - 1, 1), nb - nf)
        want_s = None if fresh else (t // nk + t) % nlev
        for j in range(lo, hi):
            if (j // nlev) % nk == want_k and (want_s is None or j % nlev == want_s):
                out.append(j)
                break
    return np.array(out, np.int64)


def cpu_baseline_leg(args, ix, cpu_q, cpu_k, gpu_d, gpu_i):
    """The reference's serial exact search (oracle/_ref/hercules, built from
    the reference sources) on a few of the timed queries, each with its own
    k, over the index files the GPU wrote.  Returns (baseline, parity,
    index digests): parity compares the reference's printed answers
    (Query_exact_distance = %f of the square root, Query_exact_node_file_pos)
    with the GPU's batched answers for the same queries and with the plain
    path's answer-leaf positions."""
    from oracle import oracle as O
    d = None
    na = {"value": None, "unit": UNIT, "cores": 1, "kind": "reference"}
    try:
        if not os.path.exists(O.REF_BIN):
            return dict(na, sample="unavailable: oracle/_ref/hercules not built"), None, None
        d = write_index_for_cpu(ix, args)
        if d is None:
            return dict(na, sample="unavailable: no host space for the index files"), None, None
        index = dict(index_digests(d), built_by="GPU (hg_index_build on the device, written by hg_index_write)",
                     digest="SHA-256 over the SHA-256 of each 64 MiB chunk")
        secs, nq, wall = 0.0, 0, 0.0
        checked, mismatches = 0, []
        for j, (q, k) in enumerate(zip(cpu_q, cpu_k)):
            k = int(k)
            per_q, w, ans = cpu_reference_run(args, d, q[None, :], threads=1, k=k)
            secs += sum(per_q.values())
            nq += len(per_q)
            wall += w
            _, _, pos = ix.knn(q[None, :], k, with_leaf_pos=True)
            want_d = ["%f" % np.sqrt(v) for v in gpu_d[j, :k]]
            want_p = [str(int(v)) for v in pos[0]]
            got = ans.get(1, {"dist": [], "pos": []})
            checked += 1
            if got["dist"] != want_d or got["pos"] != want_p:
                mismatches.append({"query": j, "k": k, "reference": got, "gpu": {"dist": want_d, "pos": want_p}})
        baseline = dict(na, value=round(nq / secs, 4) if secs > 0 else None,
                        sample="%d of the timed queries (k = %s), reference exact_de_knn_search (--num-threads 1) "
                               "over the same %dx%d index files; per-query time from its Query_total_time_secs; "
                               "wall %.1f s" % (nq, ",".join(str(int(k)) for k in cpu_k), args.n, args.L, wall))
        parity = {"ref_queries": checked, "k": [int(k) for k in cpu_k], "match": not mismatches,
                  "what": "reference CLI's printed distances and answer-leaf file positions == the GPU batched "
                          "path's distances (%f of the square root) and the plain path's answer leaves",
                  "mismatches": mismatches[:3]}
        return baseline, parity, index
    except Exception as e:  # the baseline is reported, never fatal
        return dict(na, sample="failed: %s" % e), {"match": None, "error": str(e)}, None
    finally:
        if d:
            shutil.rmtree(d, ignore_errors=True)


def host_index_dir(need_bytes, prefix):
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(base)
            if st.f_bavail * st.f_frsize > need_bytes:
                return tempfile.mkdtemp(prefix=prefix, dir=base) + "/"
        except OSError:
            continue
    return None


def run_reference(args, rank, world, local):
    """--impl reference: the reference's multi-threaded query path on the
    host cores, on queries of the timed batches (each with its own k).  This
    process maps nothing of hercules_b200: the collection and the queries
    come from the oracle's restatement of the generator (the same bits as
    the GPU's), the index files from the oracle's restatement of the
    reference's one-worker build (byte-identical to the reference's own
    build, as the tests check), written on every host core."""
    if rank != 0:
        return
    from oracle import oracle as O
    if not os.path.exists(O.REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/hercules was not built from the "
                                                               "reference sources"}))
        return
    threads = os.cpu_count() or 1
    nps = args.ref_queries_per_step
    t0 = time.perf_counter()
    d = host_index_dir(args.n * args.L * 4 * 1.05 + (1 << 30), "hg_ref_idx_")
    if d is None:
        print(json.dumps({"impl": "reference", "unavailable": "no host space for the %d x %d index files"
                                                               % (args.n, args.L)}))
        return
    try:
        X = O.gen_rows(DATA_SEED, args.n, args.L, unit=args.data == "unit")
        oi = O.OracleIndex.build_mt(X, args.leaf, keep_rows=False)
        oi.write(d, 64.0)
        del oi, X
        setup_s = time.perf_counter() - t0
        index = dict(index_digests(d), built_by="oracle restatement of the reference's one-worker build "
                                                "(or_build_mt), on the host", digest="SHA-256 over the SHA-256 "
                                                                                     "of each 64 MiB chunk")
        # --sax-threshold above 1 keeps the reference on its serial refine
        # branch: its threaded refine worker never advances and hangs
        # (hercules_query_engine.c:1987-2026)
        extra = ("--sims", "--eapca-threshold", "0.25", "--sax-threshold", "1.1")
        times, wall, ks_used = [], 0.0, []
        for step in range(args.warmup + args.steps):
            Qh, ks = batch_on_host(args, O, step)
            # nps positions of this step's batch, rotating so that the
            # steps together cover every (sigma^2, k) pair and the fresh walks
            pos = [(step * 131 + t * args.batch // nps) % args.batch for t in range(nps)]
            for j in pos:
                per_q, w, _ = cpu_reference_run(args, d, Qh[j][None, :], threads=threads, extra=extra, k=int(ks[j]))
                times.append((step, sum(per_q.values())))
                wall += w
                if step >= args.warmup:
                    ks_used.append(int(ks[j]))
        timed = [t for st, t in times if st >= args.warmup]
        secs = sum(timed)
        value = len(timed) / secs if secs > 0 else None
        sample = ("%d queries per step from that step's batch of the workload (k used: %s); reference "
                  "--num-threads %d --sims --eapca-threshold 0.25 --sax-threshold 1.1 over index files built by "
                  "the oracle on the host; per-query time from its Query_total_time_secs; wall %.1f s, "
                  "setup %.1f s" % (nps, ",".join(map(str, sorted(set(ks_used)))), threads, wall, setup_s))
        line = {"impl": "reference", "metric": METRIC, "value": round(value, 4) if value else None, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * secs / max(args.steps, 1), "higher_is_better": True,
                "scaling": "strong" if world > 1 and args.multi == "shard" else "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded z-normalised random walks; "
                                                             "noisy and fresh queries)",
                "config": config_of(args),
                "cpu_baseline": {"value": round(value, 4) if value else None, "unit": UNIT, "cores": threads,
                                 "kind": "reference", "sample": sample},
                "e2e": {"value": round(value, 4) if value else None, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0},
                "index": index}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
