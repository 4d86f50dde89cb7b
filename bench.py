#!/usr/bin/env python
"""bench.py -- exact k-NN queries/s on one B200 at 25M x 256 (Hercules path).

Workload (default): 25,000,000 z-normalised random walks of length 256
(25.6 GB float32, resident in HBM; seeded synthetic data, dataset seed 1184),
leaf size 100,000, exact k-NN with k = 10 for noisy queries (a random dataset
series plus N(0, sigma^2) noise, sigma^2 cycling 0.01 / 0.1 / 1.0, query seed
14784).  A step is one batch of --queries-per-step queries through the plain
per-query path (hg_knn_device); `value` is queries per second over the timed
steps with the collection already in HBM; `e2e` is the same through hg_knn
with the queries in pinned host memory and results copied back every step.

The data (25.6 GB) is far larger than L2 (126 MB); every query streams from
HBM, so no L2 flush is needed between steps.

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

METRIC = "exact k-NN queries/s @25Mx256"
UNIT = "queries/s"
DATA_SEED = 1184
QUERY_SEED = 14784


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--n", type=int, default=25_000_000)
    p.add_argument("--L", type=int, default=256)
    p.add_argument("--leaf", type=int, default=100_000)
    p.add_argument("--k", type=int, default=10)
    p.add_argument("--queries-per-step", type=int, default=64)
    p.add_argument("--lb-sax", type=int, default=1)
    p.add_argument("--cpu-sample-queries", type=int, default=3)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--ref-queries-per-step", type=int, default=2)
    return p.parse_args()


def sigma2_for(nq, offset=0):
    cyc = np.array([0.01, 0.1, 1.0])
    return cyc[(np.arange(nq) + offset) % 3]


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


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("gloo" if args.impl == "reference" else "nccl",
                                timeout=datetime.timedelta(seconds=600))
    return rank, world, local


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


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """DRAM traffic per algorithmic byte of the distance kernel, from the
    committed ncu summary (profiles/k_ed_stream_traffic.json)."""
    p = os.path.join(ROOT, "profiles", "k_ed_stream_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        return json.load(open(p))
    except ValueError:
        return None


def build_collection(args, torch, H, device):
    n, L = args.n, args.L
    X = torch.empty((n, L), dtype=torch.float32, device=device)
    H.generate_walks_device(DATA_SEED, n, L, X.data_ptr(), device=device)
    torch.cuda.synchronize()
    return X


def make_queries(args, torch, H, X, nq, device, offset):
    Q = torch.empty((nq, args.L), dtype=torch.float32, device=device)
    H.generate_queries_device(QUERY_SEED + offset, X.data_ptr(), args.n, args.L, sigma2_for(nq), Q.data_ptr(),
                              device=device)
    torch.cuda.synchronize()
    return Q


def cpu_reference_run(args, index_dir, queries_host, threads, extra=()):
    """Runs the reference CLI over the written index; per-query seconds from
    its own Query_total_time_secs lines."""
    from oracle import oracle as O
    binary = O.REF_BIN
    qfile = os.path.join(index_dir, "bench_queries.bin")
    np.ascontiguousarray(queries_host, np.float32).tofile(qfile)
    nq = queries_host.shape[0]
    cmd = [binary, "--mode", "1", "--serial", "1", "--num-threads", str(threads), "--k", str(args.k),
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
    nq_step = args.queries_per_step
    steps, warm = args.steps, args.warmup
    t_setup = time.perf_counter()
    X = build_collection(args, torch, H, device)
    Q = make_queries(args, torch, H, X, (steps + warm) * nq_step, device, offset=rank * 7919)
    Qe = make_queries(args, torch, H, X, (steps + warm) * nq_step, device, offset=rank * 7919 + 1)
    t0 = time.perf_counter()
    ix = H.HerculesIndex.build_device(X.data_ptr(), args.n, args.L, args.leaf, device=device)
    build_s = time.perf_counter() - t0
    cpu_q = Q[:args.cpu_sample_queries].cpu().numpy() if (rank == 0 and world == 1) else None
    del X
    torch.cuda.empty_cache()
    setup_s = time.perf_counter() - t_setup
    k = args.k
    D = torch.empty((nq_step, k), dtype=torch.float32, device=device)
    I = torch.empty((nq_step, k), dtype=torch.int64, device=device)
    stream = torch.cuda.current_stream().cuda_stream

    def step(i, profile):
        return ix.knn_device(Q[i * nq_step:(i + 1) * nq_step].data_ptr(), nq_step, k, D.data_ptr(), I.data_ptr(),
                             stream=stream, use_lb_sax=bool(args.lb_sax), profile=profile)

    for i in range(warm):
        step(i, False)
    torch.cuda.synchronize()
    barrier(world)
    clocks = ClockSampler(device)
    clocks.start()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    agg = {}
    for i in range(warm, warm + steps):
        st = step(i, True)
        for kk, v in st.items():
            agg[kk] = agg.get(kk, 0) + v
    e1.record()
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = e0.elapsed_time(e1)
    ms = max_over_ranks(ms, world, device=torch.device("cuda", device))
    total_q = nq_step * steps * world
    value = total_q / (ms / 1000.0)

    # end to end: host queries (pinned) in, host results out, every step
    Qh = torch.empty((nq_step * (steps + warm), args.L), dtype=torch.float32, pin_memory=True)
    Qh.copy_(Qe.cpu())
    Qhn = Qh.numpy()
    for i in range(warm):
        ix.knn(Qhn[i * nq_step:(i + 1) * nq_step], k, use_lb_sax=bool(args.lb_sax))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(warm, warm + steps):
        ix.knn(Qhn[i * nq_step:(i + 1) * nq_step], k, use_lb_sax=bool(args.lb_sax))
    torch.cuda.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, device=torch.device("cuda", device))
    e2e_value = total_q / e2e_s

    # roofline of the dominant kernel, the distance stream k_ed_stream:
    # algorithmic bytes = 32 B per 8-float chunk whose distance it computed
    # + 4 B list entry per row started + 8 B id per finished row, divided by
    # its summed launch time (CUDA events around every launch)
    peak, peak_kind = measured_peaks()
    launches = int(agg["scan_launches"])
    alg_bytes = 32.0 * agg["chunks_loaded"] + 4.0 * agg["rows_visited"] + 8.0 * agg["rows_completed"]
    scan_s = agg["scan_ms"] / 1000.0
    achieved = alg_bytes / scan_s / 1e9 if scan_s > 0 else 0.0
    tr = ncu_traffic()
    traffic = None
    if tr and tr.get("dram_bytes_per_algorithmic_byte"):
        # ncu traffic of a small capture, scaled to a 25M launch by its
        # algorithmic bytes (traffic grows in proportion)
        traffic = tr["dram_bytes_per_algorithmic_byte"] * alg_bytes / max(launches, 1)
    f_launches = int(agg["filter_launches"])
    f_bytes = 16.0 * agg["rows_considered"] + 4.0 * (agg["rows_considered"] - agg["rows_lbsax_pruned"])
    f_s = agg["filter_ms"] / 1000.0
    roofline = {"bound": "hbm", "kernel": "k_ed_stream", "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": peak_kind, "traffic": traffic,
                "algorithmic_bytes_per_launch": alg_bytes / max(launches, 1),
                "avg_launch_ms": agg["scan_ms"] / max(launches, 1), "launches": launches,
                "second_kernel": {"kernel": "k_lbsax_filter",
                                  "achieved": round(f_bytes / f_s / 1e9, 1) if f_s > 0 else None,
                                  "frac": round(f_bytes / f_s / 1e9 / peak, 4) if f_s > 0 else None,
                                  "avg_launch_ms": agg["filter_ms"] / max(f_launches, 1), "launches": f_launches}}

    cpu_baseline = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu_baseline = cpu_baseline_leg(args, ix, cpu_q)
    ix.close()
    # per query: prep, leaf LB, distances (approximate leaf), merge, sort,
    # LB_SAX filter, distances (candidates), merge, emit
    per_query_launches = 9
    line = {
        "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": steps, "warmup": warm,
        "ms_per_step": ms / steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded z-normalised random walks; noisy queries)",
        "config": {"workload": "plain per-query exact k-NN, %d x %d float32, leaf %d, k=%d, %d queries/step, "
                               "sigma2 0.01/0.1/1.0" % (args.n, args.L, args.leaf, k, nq_step),
                   "n": args.n, "L": args.L, "leaf_size": args.leaf, "k": k, "queries_per_step": nq_step,
                   "lb_sax": bool(args.lb_sax), "l2": "inputs (25.6 GB) larger than L2; no flush needed",
                   "parallelism": "replica per GPU" if world > 1 else "single GPU"},
        "e2e": {"value": round(e2e_value, 2), "unit": UNIT, "h2d_bytes_per_step": nq_step * args.L * 4,
                "d2h_bytes_per_step": nq_step * k * (4 + 8)},
        "gpu_launches": per_query_launches * nq_step * steps,
        "roofline": roofline,
        "cpu_baseline": cpu_baseline,
        "clocks": ck,
        "stats": {"candidate_rows_per_query": agg["rows_considered"] / (nq_step * steps),
                  "lbsax_pruned_frac": agg["rows_lbsax_pruned"] / max(agg["rows_considered"], 1),
                  "distance_rows_per_query": agg["rows_visited"] / (nq_step * steps),
                  "chunks_per_distance_row": agg["chunks_loaded"] / max(agg["rows_visited"], 1),
                  "leaves_scanned_per_query": agg["leaves_scanned"] / (nq_step * steps),
                  "ed_share_of_step": agg["scan_ms"] / ms if ms > 0 else None,
                  "filter_share_of_step": agg["filter_ms"] / ms if ms > 0 else None,
                  "index_build_s": round(build_s, 2), "setup_s": round(setup_s, 2)},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def cpu_baseline_leg(args, ix, cpu_q):
    """The reference's serial exact search (oracle/_ref/hercules, built from
    the reference sources) on a few of the same queries over the same index."""
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
        per_q, wall = cpu_reference_run(args, d, cpu_q, threads=1)
        secs = sum(per_q.values())
        return {"value": round(len(per_q) / secs, 4) if secs > 0 else None, "unit": UNIT, "cores": 1,
                "kind": "reference",
                "sample": "%d of the timed queries, reference exact_de_knn_search (--num-threads 1) over the "
                          "same %dx%d index; per-query time from its Query_total_time_secs; wall %.1f s"
                          % (len(per_q), args.n, args.L, wall)}
    except Exception as e:  # the baseline is reported, never fatal
        return {"value": None, "unit": UNIT, "cores": 1, "kind": "reference", "sample": "failed: %s" % e}
    finally:
        if d:
            shutil.rmtree(d, ignore_errors=True)


def run_reference(args, rank, world, local):
    """--impl reference: the reference's multi-threaded query path on the
    host cores over the same index files."""
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
    Q = make_queries(args, torch, H, X, (args.steps + args.warmup) * nps, local, offset=0)
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
        per_q, wall = cpu_reference_run(args, d, Q.cpu().numpy(), threads=threads, extra=extra)
        qs = sorted(per_q)
        timed = qs[args.warmup * nps:]
        secs = sum(per_q[q] for q in timed)
        value = len(timed) / secs if secs > 0 else None
        line = {"impl": "reference", "metric": METRIC, "value": round(value, 4) if value else None, "unit": UNIT,
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1000.0 * secs / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded z-normalised random walks)",
                "config": {"workload": "plain per-query exact k-NN, %d x %d float32, leaf %d, k=%d"
                                       % (args.n, args.L, args.leaf, args.k), "queries_per_step": nps},
                "cpu_baseline": {"value": round(value, 4) if value else None, "unit": UNIT, "cores": threads,
                                 "kind": "reference",
                                 "sample": "%d queries per step; reference --num-threads %d --sims "
                                           "--eapca-threshold 0.25 --sax-threshold 1.1 over the index files "
                                           "(built on the GPU, byte-identical to the reference's); wall %.1f s"
                                           % (nps, threads, wall)},
                "e2e": {"value": round(value, 4) if value else None, "unit": UNIT, "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(d, ignore_errors=True)


if __name__ == "__main__":
    main()
