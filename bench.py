#!/usr/bin/env python
"""bench.py -- exact k-NN queries/s on one B200 at 25M x 256 (Hercules path).

Collection: 25,000,000 z-normalised random walks of length 256 (25.6 GB
float32 resident in HBM; seeded synthetic data, dataset seed 1184), leaf
size 100,000, built into the Hercules EAPCA index on the GPU.

Headline workload (a step): one batch of 4,096 queries answered exactly by
the batched path (hg_knn_batch_device): equal thirds of noisy queries (a
random dataset series plus N(0, sigma^2) noise, sigma^2 = 0.01 / 0.1 / 1.0,
z-normalised) plus 10% fresh random walks, k cycling 1 / 10 / 100.  `value`
is queries per second over the timed steps (CUDA events on the stream, the
collection and the step's queries already in HBM); `e2e` is the same through
hg_knn_batch with the queries in pinned host memory and the answers copied
back every step.  The plain per-query path (hg_knn_device, k = 10) is timed
beside it on the same collection (`plain`), with the leaf-scan kernel's
HBM roofline (`leaf_scan`), and so is the unindexed full scan (`pscan`,
HG_MODE_PSCAN) with the reference's multi-threaded CPU PSCAN on a bounded
sample beside it.  `fp64_oracle` checks a timed batch's answers against an
FP64 brute force over the whole collection; `certified_bound` reports the
filter's error bound.

The BF16 copy of the collection (12.8 GB) and the raw rows (25.6 GB) are far
larger than L2 (126 MB); every step streams them from HBM, so no L2 flush is
needed between steps.

--impl reference runs the reference Hercules query path (oracle/_ref/hercules,
compiled from the reference's own sources) on the host cores over the same
index files, which the GPU build writes byte-identical to the reference's.

Multi-GPU (torchrun): every rank holds a full replica of the collection and
answers its own queries; there is no data-path collective (weak scaling).
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
    p.add_argument("--plain-queries", type=int, default=128, help="queries through the plain path")
    p.add_argument("--plain-k", type=int, default=10)
    p.add_argument("--data", choices=["walks", "unit"], default="walks",
                   help="z-normalised random walks, or unit-normalised Gaussian vectors")
    p.add_argument("--sigma2", default="0.01,0.1,1.0", help="noise levels of the noisy queries, in equal shares")
    p.add_argument("--ks", default="1,10,100", help="k of the batched queries, cycling")
    p.add_argument("--cpu-sample-queries", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-queries-per-step", type=int, default=2)
    p.add_argument("--no-autotune", action="store_true", help="keep the default launch parameters")
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
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
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


def make_batches(args, torch, H, X, nbatches, device, offset):
    """nbatches batches of args.batch queries: noisy queries (sigma^2 in
    equal thirds) followed by fresh random walks (args.fresh_frac)."""
    nb = args.batch
    nf = int(round(nb * args.fresh_frac))
    Q = torch.empty((nbatches, nb, args.L), dtype=torch.float32, device=device)
    gen = H.generate_unit_queries_device if args.data == "unit" else H.generate_queries_device
    fresh = H.generate_unit_vectors_device if args.data == "unit" else H.generate_walks_device
    for i in range(nbatches):
        gen(QUERY_SEED + offset + i, X.data_ptr(), args.n, args.L, sigma2_for(nb - nf, levels=levels_of(args)),
            Q[i].data_ptr(), device=device)
        if nf:
            fresh(FRESH_SEED + offset, nf, args.L, Q[i, nb - nf:].data_ptr(), first=(offset + i) * nf, device=device)
    torch.cuda.synchronize()
    kc = ks_of(args)
    ks = np.array(kc, np.uint32)[np.arange(nb) % len(kc)]
    return Q, ks


def fp64_oracle_check(args, torch, H, Q, ks, D, I, device, nsample=32):
    """FP64 brute force over the whole collection (regenerated chunk by chunk
    from the same seed) for the first nsample queries of a timed batch:
    recall of the returned ids against the FP64 k nearest, and the relative
    error of the returned FP32 distances against the FP64 distances of the
    same rows."""
    s = min(nsample, Q.shape[0])
    n, L = args.n, args.L
    q = Q[:s].double()
    kq = torch.as_tensor(ks[:s].astype(np.int64), device=q.device)
    kmax = int(kq.max())
    ours = I[:s, :kmax]
    ours_d = D[:s, :kmax].double()
    gen = H.generate_unit_vectors_device if args.data == "unit" else H.generate_walks_device
    chunk = max(1, min(n, (1 << 28) // L))
    buf = torch.empty((chunk, L), dtype=torch.float32, device=device)
    best_d = torch.full((s, kmax), float("inf"), dtype=torch.float64, device=device)
    best_i = torch.full((s, kmax), -1, dtype=torch.int64, device=device)
    d64_ours = torch.full((s, kmax), float("nan"), dtype=torch.float64, device=device)
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
    hits, total, max_rel = 0, 0, 0.0
    for j in range(s):
        k = int(kq[j])
        a = set(ours[j, :k].tolist())
        b = set(best_i[j, :k].tolist())
        hits += len(a & b)
        total += k
        d64 = d64_ours[j, :k]
        rel = ((ours_d[j, :k] - d64).abs() / d64.clamp_min(1e-30)).max()
        max_rel = max(max_rel, float(rel))
    return {"queries": s, "pairs": total, "recall_vs_fp64_topk": round(hits / max(total, 1), 6),
            "max_rel_err_vs_fp64": max_rel,
            "how": "FP64 brute force over all %d rows, regenerated from the data seed in chunks" % n}


def cpu_reference_run(args, index_dir, queries_host, threads, extra=(), k=10):
    """Runs the reference CLI over the written index; per-query seconds from
    its own Query_total_time_secs lines."""
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
    per_q = {}
    for line in r.stdout.splitlines():
        parts = line.split("\t")
        if len(parts) == 5 and parts[0] == "Query_total_time_secs":
            per_q.setdefault(int(parts[3]), 0.0)
            per_q[int(parts[3])] += float(parts[1])
    return per_q, wall


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
    need = args.n * args.L * 4 * 1.3
    for base in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(base)
            if st.f_bavail * st.f_frsize > need:
                d = tempfile.mkdtemp(prefix="hg_bench_idx_", dir=base) + "/"
                ix.write(d, buffer_mb=64.0)
                return d
        except OSError:
            continue
    return None


def main():
    args = parse()
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, rank, world, local)
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
    cpu_q = Qb[0, :args.cpu_sample_queries].cpu().numpy() if (rank == 0 and world == 1) else None
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

    # answers of the last timed batch against an FP64 brute force
    fp64 = fp64_oracle_check(args, torch, H, Qb[warm + steps - 1], ks, D, I, device)

    # the plain per-query path on the same collection, every scan launch timed
    pk = args.plain_k
    Dp = torch.empty((args.plain_queries, pk), dtype=torch.float32, device=device)
    Ip = torch.empty((args.plain_queries, pk), dtype=torch.int64, device=device)
    ix.knn_device(Qp.data_ptr(), min(8, args.plain_queries), pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream,
                  use_lb_sax=True)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    pst = ix.knn_device(Qp.data_ptr(), args.plain_queries, pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream,
                        use_lb_sax=True, profile=True)
    p1.record()
    torch.cuda.synchronize()
    plain_ms = p0.elapsed_time(p1)
    plain_qps = args.plain_queries / (plain_ms / 1000.0)

    # PSCAN (every row of the collection per query, HG_MODE_PSCAN): the
    # unindexed baseline, HBM-bound
    npq = max(1, min(4, args.plain_queries))
    ix.knn_device(Qp.data_ptr(), 1, pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream, mode=H.MODE_PSCAN)
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0.record()
    sst = ix.knn_device(Qp.data_ptr(), npq, pk, Dp.data_ptr(), Ip.data_ptr(), stream=stream, mode=H.MODE_PSCAN,
                        profile=True)
    s1.record()
    torch.cuda.synchronize()
    pscan_ms = s0.elapsed_time(s1)
    pscan_bytes = 32.0 * sst["chunks_loaded"] + 8.0 * sst["rows_completed"]
    pscan_scan_s = (sst["scan_ms"] if sst["scan_ms"] > 0 else pscan_ms) / 1000.0
    pscan_gbs = pscan_bytes / pscan_scan_s / 1e9
    pscan = {"value": round(npq / (pscan_ms / 1000.0), 2), "unit": UNIT, "queries": npq, "k": pk,
             "path": "hg_knn_device, HG_MODE_PSCAN (every row, early abandon at the running k-th distance)",
             "scan": {"kernel": "k_ed_stream", "achieved": round(pscan_gbs, 1), "unit": "GB/s",
                      "frac": round(pscan_gbs / measured_peaks_all()["hbm"], 4),
                      "algorithmic_bytes_per_query": pscan_bytes / npq}}

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_baseline = cpu_baseline_leg(args, ix, cpu_q, ks[:args.cpu_sample_queries])
        pscan["cpu_baseline"] = cpu_pscan_leg(args, H, Qp[:npq].cpu().numpy(), pk)
    ix.close()

    # roofline of the dominant kernel, the tensor-core filter k_umma_filter:
    # algorithmic FLOPs = 2 L per (query, row) pair it evaluated, over its
    # summed launch time (CUDA events around every launch)
    peaks = measured_peaks_all()
    gemm_s = agg["gemm_ms"] / 1000.0
    flops = 2.0 * args.L * agg["bf16_pairs"]
    achieved_tf = flops / gemm_s / 1e12 if gemm_s > 0 else 0.0
    filt_launches = steps  # one full filter pass per step, plus retry rounds on a few queries
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
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16 filter (fp32 accumulate) + f32 exact re-rank",
        "data": "synthetic (seeded z-normalised random walks; noisy and fresh queries)",
        "config": {"workload": "batched exact k-NN, %d x %d float32 %s, leaf %d, %d queries/step, k cycling %s, "
                               "sigma2 in equal shares %s + %d%% fresh %s"
                               % (args.n, args.L, "z-normalised random walks" if args.data == "walks" else
                                  "unit-normalised Gaussian vectors", args.leaf, nb, "/".join(map(str, ks_of(args))),
                                  "/".join(map(str, levels_of(args))), int(round(100 * args.fresh_frac)),
                                  "walks" if args.data == "walks" else "vectors"),
                   "n": args.n, "L": args.L, "leaf_size": args.leaf, "queries_per_step": nb, "k": list(ks_of(args)),
                   "data": args.data,
                   "l2": "inputs (%.1f GB f32 + %.1f GB bf16) larger than L2; no flush needed"
              % (args.n * args.L * 4 / 1e9, args.n * args.L * 2 / 1e9),
                   "parallelism": "replica per GPU" if world > 1 else "single GPU",
                   "tuning": {k: tuning[k] for k in ("filter_tiles_per_item", "bound_tiles_per_item",
                                                     "rerank_blocks_per_sm", "approx_blocks_per_sm")},
                   "tuned": not args.no_autotune},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": nb * args.L * 4,
                "d2h_bytes_per_step": nb * kmax * (4 + 8)},
        "gpu_launches": int(agg["kernel_launches"]),
        "roofline": roofline,
        "leaf_scan": leaf_scan,
        "plain": {"value": round(plain_qps, 2), "unit": UNIT, "queries": args.plain_queries, "k": pk,
                  "path": "hg_knn_device (one query at a time, LB_SAX on)",
                  "batched_over_plain": round(value / plain_qps, 2) if plain_qps > 0 else None},
        "cpu_baseline": cpu_baseline,
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


def cpu_baseline_leg(args, ix, cpu_q, cpu_k):
    """The reference's serial exact search (oracle/_ref/hercules, built from
    the reference sources) on a few of the timed queries, each with its own
    k, over the same index."""
    from oracle import oracle as O
    d = None
    try:
        if not os.path.exists(O.REF_BIN):
            return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                    "sample": "unavailable: oracle/_ref/hercules not built"}
        d = write_index_for_cpu(ix, args)
        if d is None:
            return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference",
                    "sample": "unavailable: no host space for the index files"}
        secs, nq, wall = 0.0, 0, 0.0
        for q, k in zip(cpu_q, cpu_k):
            per_q, w = cpu_reference_run(args, d, q[None, :], threads=1, k=int(k))
            secs += sum(per_q.values())
            nq += len(per_q)
            wall += w
        return {"value": round(nq / secs, 4) if secs > 0 else None, "unit": UNIT, "cores": 1,
                "kind": "reference",
                "sample": "%d of the timed queries (k = %s), reference exact_de_knn_search (--num-threads 1) over "
                          "the same %dx%d index; per-query time from its Query_total_time_secs; wall %.1f s"
                          % (nq, ",".join(str(int(k)) for k in cpu_k), args.n, args.L, wall)}
    except Exception as e:  # the baseline is reported, never fatal
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "failed: %s" % e}
    finally:
        if d:
            shutil.rmtree(d, ignore_errors=True)


def run_reference(args, rank, world, local):
    """--impl reference: the reference's multi-threaded query path on the
    host cores over the same index files, on queries of the batched
    workload (each with its own k)."""
    if rank != 0:
        return
    from oracle import oracle as O
    if not os.path.exists(O.REF_BIN):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/hercules was not built from the "
                                                               "reference sources"}))
        return
    import torch
    import hercules_b200 as H
    from hercules_b200 import build as B
    B.build()
    torch.cuda.set_device(local)
    nps = args.ref_queries_per_step
    X = build_collection(args, torch, H, local)
    Qb, ks = make_batches(args, torch, H, X, 1, local, offset=0)
    ix = H.HerculesIndex.build_device(X.data_ptr(), args.n, args.L, args.leaf, device=local)
    del X
    torch.cuda.empty_cache()
    d = write_index_for_cpu(ix, args)
    ix.close()
    if d is None:
        print(json.dumps({"impl": "reference", "unavailable": "no host space for the %d x %d index files"
                                                               % (args.n, args.L)}))
        return
    try:
        threads = os.cpu_count() or 1
        # --sax-threshold above 1 keeps the reference on its serial refine
        # branch: its threaded refine worker never advances and hangs
        # (hercules_query_engine.c:1987-2026)
        extra = ("--sims", "--eapca-threshold", "0.25", "--sax-threshold", "1.1")
        total = (args.steps + args.warmup) * nps
        # spread the sample over the batch so the noise levels, fresh walks
        # and k values appear in the batch's proportions
        pick = np.linspace(0, args.batch - 1, total).astype(np.int64)
        Qh = Qb[0].cpu().numpy()
        times, wall = [], 0.0
        for j in pick:
            per_q, w = cpu_reference_run(args, d, Qh[j][None, :], threads=threads, extra=extra, k=int(ks[j]))
            times.append(sum(per_q.values()))
            wall += w
        timed = times[args.warmup * nps:]
        secs = sum(timed)
        value = len(timed) / secs if secs > 0 else None
        line = {"impl": "reference", "metric": METRIC, "value": round(value, 4) if value else None, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * secs / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded z-normalised random walks)",
                "config": {"workload": "batched exact k-NN workload, %d x %d float32, leaf %d, k cycling 1/10/100, "
                                       "queries answered one at a time by the reference" % (args.n, args.L, args.leaf),
                           "queries_per_step": nps},
                "cpu_baseline": {"value": round(value, 4) if value else None, "unit": UNIT, "cores": threads,
                                 "kind": "reference",
                                 "sample": "%d queries per step spread over a batch of the workload; reference "
                                           "--num-threads %d --sims --eapca-threshold 0.25 --sax-threshold 1.1 "
                                           "over the index files (built on the GPU, byte-identical to the "
                                           "reference's); wall %.1f s" % (nps, threads, wall)},
                "e2e": {"value": round(value, 4) if value else None, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
