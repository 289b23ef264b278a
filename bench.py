"""Benchmark of the sparse-search hot path, queries per second.

Default workload (`--workload sq8-8.8m`, the headline): SEISMIC-SQ search with
8-bit codes (per-index min/max scale) over 8,800,000 synthetic docs (the shape
of MS MARCO SPLADE: lognormal nnz median 120 over the 30,522-term BERT vocab,
Zipf(1.1) terms, lognormal(0, 0.8) values; seeded, not the dataset), built on
the GPU with lambda=6000, beta=600, alpha=0.4, seed=7; 65,536 queries of 5-200
terms per step in four launches of 16,384; cut 12, heap factor 0.9, k=10.
`value` times the device-resident step (CUDA-graph replays, queries and
results in HBM); `e2e` times the same queries through `Index.search` with host
buffers (copies inside the timed region). The index (~4 GB) exceeds L2, and L2
is also flushed between timed steps.

Other workloads: `fp32-1m` (SEISMIC fp32, 1M docs, 10,000 queries, lambda 4000,
beta 400, alpha 0.4, cut 10, heap factor 0.8), `brutal-100k` (exact brute
force), `build-1m` (the device build beside the reference's GPU-offload build).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  python bench.py --docs 3000000 --queries 16384 --kernel-only --no-graph --variant 4
      (a smaller case of the headline, search launches only: the profiling
      case; --variant/--tuning pick the search kernel)

Under torchrun each rank is a replica holding the whole index and searching
its own queries (weak scaling, no collective on the data path).
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for p in (os.path.join(ROOT, "neural-sparse-cpp_b200", "python"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

N_DOCS = 1_000_000
N_QUERIES = 10_000
SPEC = "seismic,lambda=4000|beta=400|alpha=0.4|seed=7"
CUT, HF, K = 10, 0.8, 10
METRIC = "QPS@recall@10 (SEISMIC fp32, batched, 1M docs)"
WORKLOAD = {"workload": "seismic_fp32_1M_docs_10k_queries", "docs": N_DOCS, "queries": N_QUERIES,
            "vocab": 30522, "lambda": 4000, "beta": 400, "alpha": 0.4, "cut": CUT,
            "heap_factor": HF, "k": K, "l2": "flushed between steps; index > L2"}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), \
        int(os.environ.get("LOCAL_RANK", "0"))


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    QUERY = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 3 + i and r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(self.rows)}


def reference_inputs():
    """The reference arm generates its inputs with the oracle's build of the
    corpus generator (the same C source), so it maps no library of the
    engine's tree."""
    from nsparse_b200 import synth
    p = os.path.join(ROOT, "oracle", "_bin", "libnsp_synth.so")
    if os.path.exists(p):
        synth.use_library(p)


def make_data(rank):
    from nsparse_b200 import synth
    docs = synth.docs_config0(N_DOCS, seed=0)
    qs = synth.queries_config0(N_QUERIES, seed=1000 + rank)
    return docs, qs


def recall_at_k(L, T):
    v = []
    for a, b in zip(L, T):
        want = set(int(x) for x in b if x >= 0)
        if want:
            v.append(len(set(int(x) for x in a if x >= 0) & want) / len(want))
    return float(np.mean(v)) if v else 1.0


def counting_pass(nsparse, idx, q, cut, hf, args, L, D):
    """The same batch searched once more as a counting pass (untimed; same
    results): its stats count each scored doc's row once per query, as the
    reference's visited set does. The kernel itself scores a doc met again in
    a later list again, so its own byte count exceeds the reference's
    algorithmic bytes by those re-read rows."""
    p = nsparse.SeismicSearchParameters(cut, hf)
    p.set_kernel(args.variant if args.variant >= 2 else 4, args.tuning)
    p.set_count_unique(True)
    Du, Lu = idx.search(q.n, q.indptr, q.indices, q.values, K, p)
    assert (Lu == L).all() and (Du == D).all(), "counting pass changed the results"
    return nsparse.last_search_stats()


def claim_order_launches(n_queries, device=None):
    """1 when a batched search of n_queries runs the engine's claim-order
    kernel before the search kernel (four or more queries per CTA; the
    one-CTA-per-query kernel keeps four 8-warp CTAs per SM), else 0."""
    import torch
    dev = torch.cuda.current_device() if device is None else device
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    return 1 if n_queries >= 4 * min(n_queries, 4 * sms) else 0


def replica_throughput(total_ms, e2e_s, n_queries, steps, e2e_steps, world, device=None):
    """Whole-job throughput of `world` replicas, each searching its own
    `n_queries` per step: every rank's time is replaced by the slowest rank's
    (max over ranks), so the job rate is world * queries / that time. Returns
    (max timed ms, queries/s, e2e queries/s); identical on every rank."""
    if world > 1:
        import torch
        import torch.distributed as dist
        t_ = torch.tensor([float(total_ms), float(e2e_s)], dtype=torch.float64, device=device)
        dist.all_reduce(t_, op=dist.ReduceOp.MAX)
        total_ms, e2e_s = float(t_[0].item()), float(t_[1].item())
    value = world * n_queries * steps / (total_ms / 1000.0)
    e2e_value = world * n_queries * e2e_steps / e2e_s
    return total_ms, value, e2e_value


def cpu_baseline(docs, qs, index_file, sample, D_eng=None, L_eng=None, gt_L=None):
    """The reference's own search (compiled from its sources, oracle/_ref), all
    host threads, on the first `sample` queries of the workload; with the
    engine's rows for the same queries, their parity with the reference's and
    the reference's recall@10 at the same knobs."""
    import oracle as O
    variant = ref_variant()
    if variant is None:
        return None
    L = O.ref_lib(variant)
    cores = os.cpu_count()
    L.ref_set_threads(cores)
    r = O.RefIndex.read(index_file, variant=variant)
    q = qs.rows(0, sample)
    r.search(q.rows(0, min(64, sample)), K, param_kind=2, cut=CUT, heap_factor=HF)  # warm
    t = time.perf_counter()
    Dr, Lr = r.search(q, K, param_kind=2, cut=CUT, heap_factor=HF)
    dt = time.perf_counter() - t
    lat = ref_per_query_latency(L, r, q, min(200, sample), cores)
    r.close()
    out = {"value": sample / dt, "unit": "queries/s", "cores": cores, "kind": "reference",
           "sample": f"{sample} of the {N_QUERIES} queries, one batched search() call, "
                     f"reference {variant} build, OMP threads={cores}",
           "per_query_1_thread": lat}
    if gt_L is not None:
        out[f"reference_recall_at_10_{variant}"] = recall_at_k(Lr, gt_L[:sample])
    if L_eng is not None and O.ref_available("generic"):
        # parity against the reference's generic build: its sequential fp32
        # sums (utils/distance.h:29-37) are the ones the engine reproduces;
        # the SIMD builds sum in another order
        G = O.ref_lib("generic")
        G.ref_set_threads(cores)
        g = O.RefIndex.read(index_file, variant="generic")
        Dg, Lg = g.search(q, K, param_kind=2, cut=CUT, heap_factor=HF)
        g.close()
        out["parity"] = dict(row_parity(D_eng[:sample], L_eng[:sample], Dg, Lg),
                             reference_build="generic (sequential fp32 sums)")
        if gt_L is not None:
            out["reference_recall_at_10"] = recall_at_k(Lg, gt_L[:sample])
    return out


def ref_per_query_latency(L, r, q, n, cores):
    """The reference's per-query latency as its residency benchmark takes it
    (benchmarks/sq_residency_bench.cpp:249-269): one thread, one search() call
    per query, wall time of each call; p50/p99 over the first n queries."""
    L.ref_set_threads(1)
    try:
        ms = []
        for i in range(n):
            one = q.rows(i, i + 1)
            t = time.perf_counter()
            r.search(one, K, param_kind=2, cut=CUT, heap_factor=HF)
            ms.append(1000.0 * (time.perf_counter() - t))
    finally:
        L.ref_set_threads(cores)
    return {"queries": n, "p50_ms": float(np.percentile(ms, 50)),
            "p99_ms": float(np.percentile(ms, 99)), "threads": 1}


def ref_variant():
    import oracle as O
    flags = open("/proc/cpuinfo").read()
    for v, need in (("avx512", "avx512bw"), ("avx2", "avx2"), ("generic", "")):
        if O.ref_available(v) and (not need or need in flags):
            return v
    return None


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle as O
    variant = ref_variant()
    if variant is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built (oracle/_ref)"}))
        return
    reference_inputs()
    docs, qs = make_data(0)
    cores = os.cpu_count()
    O.ref_lib(variant).ref_set_threads(cores)
    t = time.perf_counter()
    r = O.RefIndex(docs.dim, SPEC, variant=variant)
    r.add(docs)
    r.build()
    build_s = time.perf_counter() - t
    log(f"reference build {build_s:.1f}s on {cores} threads")
    sample = min(2000, qs.n)  # queries per step: ~10-30 s of CPU work at the full workload
    q = qs.rows(0, sample)
    for _ in range(args.warmup):
        r.search(q.rows(0, min(200, sample)), K, param_kind=2, cut=CUT, heap_factor=HF)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        r.search(q, K, param_kind=2, cut=CUT, heap_factor=HF)
        times.append(time.perf_counter() - t)
    value = sample * len(times) / sum(times)
    lat = ref_per_query_latency(O.ref_lib(variant), r, q, min(200, sample), cores)
    out = {"metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": 0, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "impl": "reference", "config": dict(WORKLOAD, sample_queries=sample),
           "build_s": build_s,
           "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "reference",
                            "sample": f"{sample} queries per step, one batched search() call, "
                                      f"reference {variant} build",
                            "per_query_1_thread": lat},
           "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def run_engine(args):
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    import nsparse
    dev = torch.device("cuda", torch.cuda.current_device())
    docs, qs = make_data(rank)

    # ---- build on the GPU
    torch.cuda.synchronize()
    t = time.perf_counter()
    idx = nsparse.index_factory(docs.dim, SPEC)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    log(f"rank {rank}: device build {build_s:.1f}s")
    params = nsparse.SeismicSearchParameters(CUT, HF)
    params.set_kernel(args.variant, args.tuning)
    tuned = None
    if args.variant < 0:
        # the engine's autotuner picks the launch shape on 2,000 queries drawn
        # apart from the timed ones (seed 999; the timed queries use 1000+)
        from nsparse_b200 import synth
        sample = synth.queries_config0(2000, seed=999)
        tuned = idx.autotune(sample.n, sample.indptr, sample.indices, sample.values, K, params)
        log(f"autotune: {tuned}")

    # ---- device-resident inputs and outputs
    d_ip = torch.from_numpy(qs.indptr).to(dev)
    d_ix = torch.from_numpy(qs.indices.view(np.int16)).to(dev)
    d_v = torch.from_numpy(qs.values).to(dev)
    d_D = torch.empty((qs.n, K), dtype=torch.float32, device=dev)
    d_L = torch.empty((qs.n, K), dtype=torch.int32, device=dev)
    max_nnz = int(np.diff(qs.indptr).max())
    # one explicit stream carries the flush, the events and the search kernel
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)

    idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)  # uploads lists
    torch.cuda.synchronize()
    graph = None
    if not args.no_graph:
        # the step captured once as a CUDA graph over these device buffers
        graph = nsparse.SearchGraph(
            idx, qs.n, qs.nnz, max_nnz, K, params,
            device_buffers={"indptr": d_ip.data_ptr(), "indices": d_ix.data_ptr(),
                            "values": d_v.data_ptr(), "distances": d_D.data_ptr(),
                            "labels": d_L.data_ptr()})

    def step():
        if graph is not None:
            graph.launch(stream.cuda_stream)
        else:
            idx.search_device(qs.n, d_ip.data_ptr(), d_ix.data_ptr(), d_v.data_ptr(), max_nnz, K,
                              d_D.data_ptr(), d_L.data_ptr(), params, stream.cuda_stream)

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    # the timed steps sit in an NVTX range ("timed"), so a profiler can take
    # exactly their launches (ncu --nvtx --nvtx-include timed/)
    with Clocks(torch.cuda.current_device()) as clk, torch.cuda.stream(stream):
        torch.cuda.nvtx.range_push("timed")
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            step()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    if graph is not None:
        graph.sync(stream.cuda_stream)  # raises if the kernel flagged an error
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"case": dict(WORKLOAD, docs=docs.n, queries=qs.n),
                              "variant": args.variant, "tuning": args.tuning,
                              "ms_per_step": total_ms / args.steps,
                              "queries_per_s": qs.n * args.steps / (total_ms / 1000.0)}))
        return
    # kernel-only time and algorithmic bytes of one batched search (engine stats)
    D, L = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)
    st = nsparse.last_search_stats()
    hD, hL = d_D.cpu().numpy(), d_L.cpu().numpy()
    assert (hL == L).all() and (hD == D).all(), "device-resident and host paths disagree"
    st_u = counting_pass(nsparse, idx, qs, CUT, HF, args, L, D)

    # ---- e2e: host buffers through the public API, copies included
    e2e_t = []
    for _ in range(args.steps):
        t = time.perf_counter()
        idx.search(qs.n, qs.indptr, qs.indices, qs.values, K, params)
        e2e_t.append(time.perf_counter() - t)
    h2d = 4 * (qs.n + 1) + 2 * qs.nnz + 4 * qs.nnz
    d2h = qs.n * K * 8
    # the same, through the captured step's host path (pinned staging)
    e2e_graph = None
    if graph is not None:
        hgraph = nsparse.SearchGraph(idx, qs.n, qs.nnz, max_nnz, K, params)
        Dg, Lg = hgraph.search(qs.n, qs.indptr, qs.indices, qs.values)
        assert (Lg == L).all() and (Dg == D).all(), "graph and ordinary search disagree"
        tg = []
        for _ in range(args.steps):
            t = time.perf_counter()
            hgraph.search(qs.n, qs.indptr, qs.indices, qs.values)
            tg.append(time.perf_counter() - t)
        hgraph.close()
        e2e_graph = {"value": qs.n * len(tg) / sum(tg), "unit": "queries/s",
                     "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}

    # ---- plain per-query path on a sample, and recall vs exact
    plain = nsparse.SeismicSearchParameters(CUT, HF)
    plain.set_engine(plain=True)
    n_plain = min(300, qs.n)
    qp = qs.rows(0, n_plain)
    idx.search(qp.rows(0, 4).n, qp.rows(0, 4).indptr, qp.rows(0, 4).indices, qp.rows(0, 4).values,
               K, plain)
    lat = []
    for q in range(n_plain):
        r1 = qp.rows(q, q + 1)
        t = time.perf_counter()
        Dp, Lp = idx.search(1, r1.indptr, r1.indices, r1.values, K, plain)
        lat.append(time.perf_counter() - t)
        assert (Lp[0] == L[q]).all()
    plain_qps = n_plain / sum(lat)
    brute = nsparse.index_factory(docs.dim, "inverted")
    brute.add(docs.n, docs.indptr, docs.indices, docs.values)
    brute.build()
    _, Lt = brute.search(qs.n, qs.indptr, qs.indices, qs.values, K)
    rec = recall_at_k(L, Lt)
    del brute

    # ---- aggregate over ranks: max time
    my_ms, value, e2e_value = replica_throughput(total_ms, sum(e2e_t), qs.n, args.steps,
                                                 len(e2e_t), world, dev)

    peak, peak_kind = measured_peaks()
    algo = st_u.reference_bytes  # each scored row once per query, over the timed kernel's time
    achieved = algo / (st.kernel_ms / 1000.0) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "seismic_search_fp32_1M.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            with tempfile.TemporaryDirectory() as td:
                fpath = os.path.join(td, "c1.idx")
                nsparse.write_index(idx, fpath)
                cpu = cpu_baseline(docs, qs, fpath, min(2000, qs.n), D, L, Lt)
        lat_ms = sorted(1000 * x for x in lat)
        out = {
            "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": my_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": dict(WORKLOAD, parallelism=f"replicas{world}",
                                                step="cuda graph replay" if graph is not None
                                                else "search_device call",
                                                kernel_variant=args.variant,
                                                kernel_tuning=args.tuning, autotuned=tuned),
            "recall_at_10": rec, "build_s": build_s,
            "plain": {"qps": plain_qps, "queries": n_plain,
                      "p50_ms": lat_ms[len(lat_ms) // 2], "p99_ms": lat_ms[int(0.99 * (len(lat_ms) - 1))],
                      "batched_over_plain": value / world / plain_qps},
            "batch_latency_ms": {"p50": statistics.median(step_ms), "max": max(step_ms)},
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "e2e_graph": e2e_graph,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": algo,
                         "bytes_read_per_launch": st.bytes,
                         "kernel_ms_per_launch": st.kernel_ms},
            "work": {"docs_scored_per_query": st.docs_scored / qs.n,
                     "unique_docs_scored_per_query": st_u.unique_docs / qs.n,
                     "blocks_visited_per_query": st.blocks_visited / qs.n},
            # per step: the claim order and the search
            "gpu_launches": args.steps * (1 + claim_order_launches(qs.n)),
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(out))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


# SEISMIC-SQ at 8.8M docs -- the hot path's target workload: uint8 codes
# (per-index min/max scale), queries of 5-200 terms, posting cap 6,000, 600
# blocks per full list, alpha 0.4, query cut 12, heap factor 0.9; 65,536
# queries per step in launches of 16,384.
SQ_DOCS = 8_800_000
SQ_QUERIES = 65_536
SQ_BATCH = 16_384
SQ_CUT, SQ_HF = 12, 0.9
SQ_QUERY_SEED, SQ_TUNE_SEED = 2000, 2001  # timed queries; the autotuner's own sample
SQ_GT_QUERIES = 1000   # recall against exact search, and the reference's parity rows
SQ_CPU_SAMPLE = 2000   # queries per reference CPU search
SQ_PLAIN = 200
SQ_METRIC = "QPS@recall@10≥0.95 batched vs per-query on 1 B200; p50/p99 ms; HBM GB/s"


def sq_spec_for(vmin, vmax):
    return (f"seismic_sq,quantizer=8bit|vmin={vmin!r}|vmax={vmax!r}|lambda=6000|beta=600|"
            f"alpha=0.4|seed=7")


def sq_data(n_docs, rank):
    from nsparse_b200 import synth
    docs = synth.docs_config2(n_docs, seed=0)
    qs = synth.queries_config2(SQ_QUERIES, seed=SQ_QUERY_SEED + 100 * rank)
    return docs, qs


def sq_workload(docs, qs, hf=SQ_HF, cut=SQ_CUT):
    return {"workload": f"seismic_sq8_{docs.n}_docs_{qs.n}_queries", "docs": docs.n,
            "nnz": int(docs.nnz), "vocab": docs.dim, "queries": qs.n, "batch": SQ_BATCH,
            "query_nnz": "uniform 5-200", "quantizer": "8bit, per-index min/max",
            "lambda": 6000, "beta": 600, "alpha": 0.4, "cut": cut, "heap_factor": hf, "k": K,
            "l2": "flushed between steps; index > L2"}


def row_parity(D, L, Dr, Lr):
    """Engine rows against the reference's rows for the same queries and
    index file: identical rows (ids, their order and scores), and separately
    the rows whose scores repeat a value (their order is the reference's
    top-k holder's, which the engine follows), the scores of docs both return
    (common-pair mismatches) and the overlap of the two result sets."""
    same = (L == Lr).all(axis=1) & (D == Dr).all(axis=1)
    tied = np.array([len(set(d[l >= 0].tolist())) < int((l >= 0).sum()) for d, l in zip(D, L)])
    same_scores = (np.sort(D, axis=1) == np.sort(Dr, axis=1)).all(axis=1)
    untied = ~tied
    mism = int(((L != Lr) | (D != Dr))[untied].any(axis=1).sum())
    pairs = pair_mism = 0
    overlap = []
    for d, l, dr, lr in zip(D, L, Dr, Lr):
        ref = {int(i): float(s) for i, s in zip(lr, dr) if i >= 0}
        mine = {int(i): float(s) for i, s in zip(l, d) if i >= 0}
        common = ref.keys() & mine.keys()
        pairs += len(common)
        pair_mism += sum(1 for i in common if ref[i] != mine[i])
        if ref:
            overlap.append(len(common) / len(ref))
    return {"rows": int(len(L)), "rows_identical_frac": float(same.mean()),
            "rows_same_scores_frac": float(same_scores.mean()),
            "untied_rows": int(untied.sum()),
            "untied_rows_identical_frac": float(same[untied].mean()) if untied.any() else 1.0,
            "score_mismatches_untied_rows": mism,
            "common_pairs": pairs, "common_pair_score_mismatches": pair_mism,
            "result_overlap": float(np.mean(overlap)) if overlap else 1.0}


def sq_exact_check(docs, qs, D, L, vmin, vmax, n):
    """Every score the engine returned for the first n queries against the
    exact integer dot product of the uint8 codes (the reference's encode,
    scalar_quantizer.h:97-101), decoded by the index's scale."""
    scale = np.float32(255.0) / (np.float32(vmax) - np.float32(vmin))

    def codes(v):
        x = (v.astype(np.float32) - np.float32(vmin)) * scale
        return np.floor(np.clip(x, 0, 255) + np.float32(0.5)).astype(np.int64)

    rng_f = np.float32(vmax) - np.float32(vmin)
    dec = np.float32(rng_f * rng_f) / np.float32(255.0 * 255.0)
    dense = np.zeros(docs.dim, np.int64)
    checked = bad = 0
    for q in range(n):
        s, e = int(qs.indptr[q]), int(qs.indptr[q + 1])
        dense[qs.indices[s:e]] = codes(qs.values[s:e])
        for d, got in zip(L[q], D[q]):
            if d < 0:
                continue
            a, b = int(docs.indptr[d]), int(docs.indptr[d + 1])
            exact = np.float32(int(np.dot(codes(docs.values[a:b]), dense[docs.indices[a:b]])))
            checked += 1
            bad += int(np.float32(exact * dec) != np.float32(got))
        dense[qs.indices[s:e]] = 0
    return {"scores_checked": checked, "scores_not_exact": bad}


def sq_reference_leg(index_file, qs, gt_L, D_eng, L_eng, cut, hf):
    """The reference's own search (compiled from its sources, oracle/_ref) of
    the index file the engine wrote. Its AVX-512 build (the fastest; it sums
    uint8 products in float): batched QPS on all host threads and per-query
    single-thread latency (cpu_baseline), and its recall@10 at the same (cut,
    heap factor). Its generic build (integer sums, as the reference's scalar
    code defines them): recall and parity with the engine's rows on the recall
    queries."""
    import oracle as O
    variant = ref_variant()
    if variant is None:
        return None, None
    L = O.ref_lib(variant)
    cores = os.cpu_count()
    L.ref_set_threads(cores)
    t = time.perf_counter()
    r = O.RefIndex.read(index_file, variant=variant)
    read_s = time.perf_counter() - t
    sample = min(SQ_CPU_SAMPLE, qs.n)
    q = qs.rows(0, sample)
    r.search(q.rows(0, 64), K, param_kind=2, cut=cut, heap_factor=hf)  # warm
    t = time.perf_counter()
    Dr, Lr = r.search(q, K, param_kind=2, cut=cut, heap_factor=hf)
    dt = time.perf_counter() - t
    n_gt = len(gt_L)
    lat = _ref_latency(L, r, q, min(200, sample), cores, cut, hf)
    r.close()
    cpu = {"value": sample / dt, "unit": "queries/s", "cores": cores, "kind": "reference",
           "sample": f"first {sample} of the {qs.n} queries, one batched search() call on the "
                     f"engine-written index file, reference {variant} build, OMP threads={cores}",
           "index_read_s": read_s, "per_query_1_thread": lat}
    ref = {f"recall_at_10_{variant}": recall_at_k(Lr[:n_gt], gt_L)}
    if O.ref_available("generic"):
        G = O.ref_lib("generic")
        G.ref_set_threads(cores)
        g = O.RefIndex.read(index_file, variant="generic")
        qg = qs.rows(0, n_gt)
        Dg, Lg = g.search(qg, K, param_kind=2, cut=cut, heap_factor=hf)
        g.close()
        ref["recall_at_10"] = recall_at_k(Lg, gt_L)
        ref["parity"] = dict(row_parity(D_eng[:n_gt], L_eng[:n_gt], Dg, Lg),
                             reference_build="generic (integer code sums)")
    else:
        ref["recall_at_10"] = ref[f"recall_at_10_{variant}"]
    return cpu, ref


def _ref_latency(L, r, q, n, cores, cut, hf):
    """Per-query latency as the reference's residency benchmark takes it
    (benchmarks/sq_residency_bench.cpp:249-269): one thread, one search()
    call per query; p50/p99 over the first n queries."""
    L.ref_set_threads(1)
    try:
        ms = []
        for i in range(n):
            one = q.rows(i, i + 1)
            t = time.perf_counter()
            r.search(one, K, param_kind=2, cut=cut, heap_factor=hf)
            ms.append(1000.0 * (time.perf_counter() - t))
    finally:
        L.ref_set_threads(cores)
    return {"queries": n, "p50_ms": float(np.percentile(ms, 50)),
            "p99_ms": float(np.percentile(ms, 99)), "threads": 1}


def run_engine_sq(args):
    """The headline: SEISMIC-SQ at 8.8M docs on the device. Device build
    (seconds); the batched search of 65,536 queries per step as four captured
    16,384-query graph steps over device-resident queries and results
    (`value`); the same through the host API with copies (`e2e`); the plain
    one-query-per-call path through the same host API; recall@10 against exact
    fp32 search and against the exact ranking of the codes; the reference's
    CPU search of the engine-written file (cpu_baseline, its recall at the same
    knobs, row parity); the serving loop's latency under Poisson arrivals."""
    import torch
    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    else:
        torch.cuda.set_device(0)
    import nsparse
    from nsparse_b200 import synth
    dev = torch.device("cuda", torch.cuda.current_device())
    n_docs = args.docs or SQ_DOCS
    t = time.perf_counter()
    docs, qs = sq_data(n_docs, rank)
    if args.queries:
        qs = qs.rows(0, min(qs.n, args.queries))
    log(f"rank {rank}: generated {docs.n} docs ({docs.nnz} nnz) in {time.perf_counter() - t:.1f}s")
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    spec = sq_spec_for(vmin, vmax)
    cut, hf = SQ_CUT, SQ_HF
    batch = min(SQ_BATCH, qs.n)
    main = rank == 0 and not args.kernel_only

    # ---- exact ground truth (rank 0): fp32 search, and the exact ranking of
    # the codes (integer scores, exact in fp32 below 2^24) -- the latter
    # separates SEISMIC's pruning from the quantizer's own loss
    gt_L = Dc = None
    n_gt = min(SQ_GT_QUERIES, qs.n)
    gt = qs.rows(0, n_gt)
    if main:
        t = time.perf_counter()
        exact = nsparse.index_factory(docs.dim, "inverted")
        exact.add(docs.n, docs.indptr, docs.indices, docs.values)
        exact.build()
        _, gt_L = exact.search(gt.n, gt.indptr, gt.indices, gt.values, K)
        del exact
        scale = np.float32(255.0) / (np.float32(vmax) - np.float32(vmin))

        def codes(v):
            x = (v.astype(np.float32) - np.float32(vmin)) * scale
            return np.floor(np.clip(x, 0, 255) + np.float32(0.5)).astype(np.float32)

        exact = nsparse.index_factory(docs.dim, "inverted")
        exact.add(docs.n, docs.indptr, docs.indices, codes(docs.values))
        exact.build()
        Dc, _ = exact.search(gt.n, gt.indptr, gt.indices, codes(gt.values), K)
        del exact
        log(f"exact ground truth {time.perf_counter() - t:.1f}s")
    rng_f = np.float32(vmax) - np.float32(vmin)
    decode = float((rng_f * rng_f) / np.float32(255.0 * 255.0))  # score per code unit

    # ---- device build
    torch.cuda.synchronize()
    t = time.perf_counter()
    idx = nsparse.index_factory(docs.dim, spec)
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    idx.build()
    torch.cuda.synchronize()
    build_s = time.perf_counter() - t
    log(f"rank {rank}: device build {build_s:.1f}s")
    params = nsparse.SeismicSearchParameters(cut, hf)
    params.set_kernel(args.variant, args.tuning)
    tuned = None
    if args.variant < 0:
        # the autotuner's sample is drawn apart from the timed queries
        tq = synth.queries_config2(4096, seed=SQ_TUNE_SEED)
        tuned = idx.autotune(tq.n, tq.indptr, tq.indices, tq.values, K, params)
        log(f"autotune: {tuned}")

    # ---- device-resident queries and results; one captured graph per batch
    d_ip = torch.from_numpy(qs.indptr).to(dev)
    d_ix = torch.from_numpy(qs.indices.view(np.int16)).to(dev)
    d_v = torch.from_numpy(qs.values).to(dev)
    d_D = torch.empty((qs.n, K), dtype=torch.float32, device=dev)
    d_L = torch.empty((qs.n, K), dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream()
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=dev)
    idx.search(64, qs.indptr[:65], qs.indices, qs.values, K, params)  # device images resident
    bounds = [(b0, min(qs.n, b0 + batch)) for b0 in range(0, qs.n, batch)]
    # per-batch row pointers rebased to the batch's first entry
    b_ip = [torch.from_numpy((qs.indptr[b0:b1 + 1] - qs.indptr[b0]).astype(np.int32)).to(dev)
            for b0, b1 in bounds]
    graphs = []
    if not args.no_graph:
        for (b0, b1), ip in zip(bounds, b_ip):
            e0 = int(qs.indptr[b0])
            nnz_b = int(qs.indptr[b1]) - e0
            mx = int(np.diff(qs.indptr[b0:b1 + 1]).max())
            graphs.append(nsparse.SearchGraph(
                idx, b1 - b0, nnz_b, mx, K, params,
                device_buffers={"indptr": ip.data_ptr(), "indices": d_ix.data_ptr() + 2 * e0,
                                "values": d_v.data_ptr() + 4 * e0,
                                "distances": d_D.data_ptr() + 4 * K * b0,
                                "labels": d_L.data_ptr() + 4 * K * b0}))
    max_nnz = int(np.diff(qs.indptr).max())

    def one_pass():
        if graphs:
            for g in graphs:
                g.launch(stream.cuda_stream)
        else:
            for (b0, b1), ip in zip(bounds, b_ip):
                e0 = int(qs.indptr[b0])
                idx.search_device(b1 - b0, ip.data_ptr(), d_ix.data_ptr() + 2 * e0,
                                  d_v.data_ptr() + 4 * e0, max_nnz, K,
                                  d_D.data_ptr() + 4 * K * b0, d_L.data_ptr() + 4 * K * b0,
                                  params, stream.cuda_stream)

    with torch.cuda.stream(stream):
        for _ in range(max(args.warmup, 3)):
            flush.zero_()
            one_pass()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    with Clocks(torch.cuda.current_device()) as clk, torch.cuda.stream(stream):
        torch.cuda.nvtx.range_push("timed")  # see run_engine
        for i in range(args.steps):
            flush.zero_()
            ev[i][0].record(stream)
            one_pass()
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    for g in graphs:
        g.sync(stream.cuda_stream)  # raises if the kernel flagged an error
    hD, hL = d_D.cpu().numpy(), d_L.cpu().numpy()
    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"case": sq_workload(docs, qs, hf, cut),
                              "variant": args.variant, "tuning": args.tuning,
                              "ms_per_step": total_ms / args.steps,
                              "queries_per_s": qs.n * args.steps / (total_ms / 1000.0)}))
        for g in graphs:
            g.close()
        if world > 1:
            torch.distributed.destroy_process_group()
        return

    # ---- one batch through the host API: the kernel's own time and its
    # algorithmic bytes (engine counters), and the same results
    q1 = qs.rows(0, batch)
    D1, L1 = idx.search(q1.n, q1.indptr, q1.indices, q1.values, K, params)
    st = nsparse.last_search_stats()
    assert (L1 == hL[:batch]).all() and (D1 == hD[:batch]).all(), \
        "device-resident and host paths disagree"
    st_u = counting_pass(nsparse, idx, q1, cut, hf, args, L1, D1)

    # ---- e2e: host buffers through the public API, copies included, the
    # same 65,536 queries per step in calls of 16,384
    host_batches = [qs.rows(b0, b1) for b0, b1 in bounds]
    e2e_t = []
    for _ in range(args.steps):
        t = time.perf_counter()
        for hb in host_batches:
            idx.search(hb.n, hb.indptr, hb.indices, hb.values, K, params)
        e2e_t.append(time.perf_counter() - t)
    h2d = 4 * (qs.n + len(bounds)) + 6 * qs.nnz
    d2h = qs.n * K * 8

    # ---- plain: one query per call through the same host API
    plain = nsparse.SeismicSearchParameters(cut, hf)
    plain.set_kernel(args.variant, args.tuning)
    plain.set_engine(plain=True)
    n_plain = min(SQ_PLAIN, qs.n)
    qp = qs.rows(0, n_plain)
    idx.search(4, qp.indptr[:5], qp.indices, qp.values, K, plain)
    lat = []
    for q in range(n_plain):
        r1 = qp.rows(q, q + 1)
        t = time.perf_counter()
        Dp, Lp = idx.search(1, r1.indptr, r1.indices, r1.values, K, plain)
        lat.append(time.perf_counter() - t)
        assert (Lp[0] == hL[q]).all() and (Dp[0] == hD[q]).all(), "plain and batched disagree"
    plain_qps = n_plain / sum(lat)

    my_ms, value, e2e_value = replica_throughput(total_ms, sum(e2e_t), qs.n, args.steps,
                                                 len(e2e_t), world, dev)
    out = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        # the reference's algorithmic bytes (each scored row once per query)
        # over the timed kernel's own time
        algo = st_u.reference_bytes
        achieved = algo / (st.kernel_ms / 1000.0) / 1e9
        traffic = None
        prof = os.path.join(ROOT, "profiles", "seismic_search_sq8_8.8M.json")
        if os.path.exists(prof) and docs.n == SQ_DOCS and batch == SQ_BATCH:
            try:
                traffic = json.load(open(prof)).get("dram_bytes_per_launch")
            except Exception:
                traffic = None
        rec = recall_at_k(hL[:n_gt], gt_L)
        got = hD[:n_gt] / decode
        hit = (got >= Dc[:, K - 1:K] - 0.5) & (hL[:n_gt] >= 0)
        lat_ms = sorted(1000 * x for x in lat)
        out = {
            "metric": SQ_METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
            "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": my_ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded; stands in for MS MARCO SPLADE)",
            "config": dict(sq_workload(docs, qs, hf, cut), parallelism=f"replicas{world}",
                           step="4 CUDA-graph replays of 16,384 queries" if graphs
                           else "4 search_device calls of 16,384 queries",
                           kernel_variant=args.variant, kernel_tuning=args.tuning,
                           autotuned=tuned),
            "recall_at_10": rec,
            "recall_at_10_vs_exact_codes": float(hit.sum() / (n_gt * K)),
            "recall_queries": n_gt,
            "exact_scores": sq_exact_check(docs, qs, hD, hL, vmin, vmax, min(200, n_gt)),
            "build_s": build_s,
            "plain": {"qps": plain_qps, "queries": n_plain, "api": "Index.search, host buffers",
                      "p50_ms": lat_ms[len(lat_ms) // 2],
                      "p99_ms": lat_ms[int(0.99 * (len(lat_ms) - 1))],
                      "batched_over_plain_same_api": e2e_value / world / plain_qps,
                      "batched_device_over_plain": value / world / plain_qps},
            "batch_latency_ms": {"p50": statistics.median(step_ms), "max": max(step_ms)},
            "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind, "traffic": traffic,
                         "algorithmic_bytes_per_launch": algo,
                         "bytes_read_per_launch": st.bytes,
                         "kernel_ms_per_launch": st.kernel_ms,
                         "launch": f"{batch} queries"},
            "work": {"docs_scored_per_query": st.docs_scored / q1.n,
                     "unique_docs_scored_per_query": st_u.unique_docs / q1.n,
                     "blocks_visited_per_query": st.blocks_visited / q1.n},
            # per batch: the query encode, the claim order and the search
            "gpu_launches": args.steps * sum(2 + claim_order_launches(b1 - b0)
                                             for b0, b1 in bounds),
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu:
            with tempfile.TemporaryDirectory() as td:
                fpath = os.path.join(td, "sq.idx")
                nsparse.write_index(idx, fpath)
                cpu, ref = sq_reference_leg(fpath, qs, gt_L, hD, hL, cut, hf)
            out["cpu_baseline"] = cpu
            out["reference_same_knobs"] = ref
        if world == 1 and not args.no_serve:
            out["serving"] = serve_sweep(nsparse, idx, docs, qs, cut, hf, args.serve_rates,
                                         slots=int(str(args.serve_slots).split(",")[0]))
    for g in graphs:
        g.close()
    if out is not None:
        print(json.dumps(out))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_reference_sq(args):
    """The reference arm of the headline: the reference's own build of the
    8.8M-doc SEISMIC-SQ index (compiled from its sources, oracle/_ref, all host
    threads), then per step one batched search() of a bounded sample of the
    same queries at the same knobs. Rank 0 alone runs it."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import oracle as O
    variant = ref_variant()
    if variant is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference library not built "
                                                            "(oracle/_ref)"}))
        return
    reference_inputs()
    docs, qs = sq_data(args.docs or SQ_DOCS, 0)
    if args.queries:
        qs = qs.rows(0, min(qs.n, args.queries))
    vmin, vmax = float(docs.values.min()), float(docs.values.max())
    cores = os.cpu_count()
    L = O.ref_lib(variant)
    L.ref_set_threads(cores)
    t = time.perf_counter()
    r = O.RefIndex(docs.dim, sq_spec_for(vmin, vmax), variant=variant)
    r.add(docs)
    r.build()
    build_s = time.perf_counter() - t
    log(f"reference build {build_s:.1f}s on {cores} threads")
    workload = sq_workload(docs, qs, SQ_HF, SQ_CUT)
    del docs
    sample = min(1000, qs.n)  # queries per step: a few seconds of CPU work
    q = qs.rows(0, sample)
    for _ in range(args.warmup):
        r.search(q.rows(0, min(200, sample)), K, param_kind=2, cut=SQ_CUT, heap_factor=SQ_HF)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        r.search(q, K, param_kind=2, cut=SQ_CUT, heap_factor=SQ_HF)
        times.append(time.perf_counter() - t)
    value = sample * len(times) / sum(times)
    lat = _ref_latency(L, r, q, min(200, sample), cores, SQ_CUT, SQ_HF)
    r.close()
    print(json.dumps({
        "metric": SQ_METRIC, "value": value, "unit": "queries/s", "n_gpus": 0,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded; stands in for MS MARCO SPLADE)", "impl": "reference",
        "config": dict(workload, sample_queries=sample,
                       sample_note=f"each step searches the first {sample} of the {qs.n} "
                                   "queries (the same query distribution)"),
        "build_s": build_s,
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": "reference",
                         "sample": f"{sample} queries per step, one batched search() call, "
                                   f"reference {variant} build, OMP threads={cores}",
                         "per_query_1_thread": lat},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def run_engine_brutal(args):
    """BrutalIndex exact search at 100k docs, 1,000 queries, k=10 (the
    CPU-runnable workload): the host-buffer API end to end, the kernel's own
    time, and the reference's CPU search of the same queries beside it."""
    import torch
    torch.cuda.set_device(0)
    import nsparse
    from nsparse_b200 import synth
    n_docs = args.docs or 100_000
    n_q = args.queries or 1000
    docs = synth.docs_config0(n_docs, seed=0)
    qs = synth.queries_config0(n_q, seed=0)
    idx = nsparse.index_factory(docs.dim, "brutal")
    idx.add(docs.n, docs.indptr, docs.indices, docs.values)
    for _ in range(max(args.warmup, 3)):
        idx.search(qs.n, qs.indptr, qs.indices, qs.values, K)
    # the postings (8 B per nonzero) fit in L2 at 100k docs: flush it before
    # every timed step
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    times, kms, nbytes, launches = [], [], [], 0
    for _ in range(args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        t = time.perf_counter()
        D, L = idx.search(qs.n, qs.indptr, qs.indices, qs.values, K)
        times.append(time.perf_counter() - t)
        st = nsparse.last_search_stats()
        kms.append(st.kernel_ms)
        nbytes.append(st.bytes)
        launches += st.launches
    value = qs.n * len(times) / sum(times)
    kernel_ms = statistics.median(kms)
    bytes_ = 4 * (docs.n + 1) + 6 * docs.nnz  # forward index read once per launch
    algo = statistics.median(nbytes)  # postings of the queries' terms, counted by the kernel
    peak, peak_src = measured_peaks()
    cpu = None
    variant = ref_variant()
    if variant is not None and not args.no_cpu:
        import oracle as O
        O.ref_lib(variant).ref_set_threads(os.cpu_count())
        r = O.RefIndex(docs.dim, "brutal", variant=variant)
        r.add(docs)
        sample = qs.rows(0, min(qs.n, 200))
        r.search(sample.rows(0, 8), K)
        t = time.perf_counter()
        r.search(sample, K)
        dt = time.perf_counter() - t
        r.close()
        cpu = {"value": sample.n / dt, "unit": "queries/s", "cores": os.cpu_count(),
               "kind": "reference",
               "sample": f"{sample.n} of the {qs.n} queries, reference {variant} build"}
    print(json.dumps({
        "metric": "QPS (BrutalIndex exact, 100k docs)", "value": value, "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": max(args.warmup, 3),
        "ms_per_step": 1000 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"brutal_fp32_{docs.n}_docs_{qs.n}_queries", "k": K,
                   "l2": "flushed between steps", "kernel": "term at a time (exact_taat_kernel)"},
        "kernel_ms_per_launch": kernel_ms,
        "kernel_queries_per_s": qs.n / (kernel_ms / 1000.0),
        "forward_index_gbs": bytes_ / (kernel_ms / 1000.0) / 1e9,
        "roofline": {"bound": "hbm", "achieved": algo / (kernel_ms / 1000.0) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": algo / (kernel_ms / 1000.0) / 1e9 / peak,
                     "peak_source": peak_src, "traffic": None,
                     "algorithmic_bytes_per_launch": algo},
        "gpu_launches": launches,
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step":
                4 * (qs.n + 1) + 6 * qs.nnz, "d2h_bytes_per_step": qs.n * K * 8},
        "cpu_baseline": cpu}))


def list_digests(path):
    """One line per posting list of an index file: a digest of its blocks
    (n_clusters, offsets, docs) and one of its summaries (term_ids, term_ptr,
    csc_cluster, csc_value)."""
    import hashlib
    import oracle as O
    rows = []
    for c in O.read_index_file(path)["lists"]:
        parts = []
        for keys in (("n_clusters", "offsets", "docs"),
                     ("term_ids", "term_ptr", "csc_cluster", "csc_value")):
            h = hashlib.sha256()
            for key in keys:
                v = c[key]
                h.update(np.ascontiguousarray(v).tobytes() if isinstance(v, np.ndarray)
                         else repr(int(v)).encode())
            parts.append(h.hexdigest()[:16])
        rows.append(" ".join(parts))
    return rows


def _sha256(path):
    import hashlib
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 24), b""):
            h.update(chunk)
    return h.hexdigest()


def run_engine_build(args):
    """SEISMIC build of the benchmark index (1M docs, lambda=4000, beta=400,
    alpha=0.4, seed 7) on the device, beside the reference's own build with
    its cuSPARSE GPU offload (oracle/_ref/libnsparse_ref_avx512_gpu.so, the
    reference's stock settings: assignment on the GPU, summaries on the CPU,
    all host threads), on the same corpus and box. The two index files are
    compared list by list."""
    import filecmp
    import torch
    torch.cuda.set_device(0)
    import nsparse
    import oracle as O
    docs, _ = make_data(0)
    out = tempfile.mkdtemp()
    ours_path, ref_path = os.path.join(out, "ours.idx"), os.path.join(out, "ref_gpu.idx")
    times = []
    for _ in range(max(args.steps, 1)):
        torch.cuda.synchronize()
        t = time.perf_counter()
        idx = nsparse.index_factory(docs.dim, SPEC)
        idx.add(docs.n, docs.indptr, docs.indices, docs.values)
        idx.build()
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t)
    nsparse.write_index(idx, ours_path)
    del idx
    if args.digest_out:
        # per posting list, short digests of its blocks (docs, offsets) and of
        # its summaries, to compare with a reference file built elsewhere
        # from the same corpus
        with open(args.digest_out, "w") as f:
            f.write("\n".join(list_digests(ours_path)))
    ref = None
    if O.ref_available("avx512_gpu") and not args.no_cpu:
        cores = os.cpu_count()
        O.ref_lib("avx512_gpu").ref_set_threads(cores)
        t = time.perf_counter()
        r = O.RefIndex(docs.dim, SPEC, variant="avx512_gpu")
        r.add(docs)
        r.build()
        ref_s = time.perf_counter() - t
        r.write(ref_path)
        r.close()
        if args.digest_out:
            with open(args.digest_out + ".reference_gpu", "w") as f:
                f.write("\n".join(list_digests(ref_path)))
        same = filecmp.cmp(ours_path, ref_path, shallow=False)
        lists_same = 1.0
        if not same:
            a, b = O.read_index_file(ours_path)["lists"], O.read_index_file(ref_path)["lists"]
            eq = [np.array_equal(x["docs"], y["docs"]) and np.array_equal(x["offsets"], y["offsets"])
                  for x, y in zip(a, b)]
            lists_same = float(np.mean(eq)) if eq else 1.0
        ref = {"seconds": ref_s, "threads": cores,
               "kind": "reference, cuSPARSE GPU offload (nsparse/gpu), AVX-512 host code",
               "index_files_identical": bool(same), "lists_identical_frac": lists_same,
               "sha256": _sha256(ref_path)}
        log(f"reference GPU-offload build {ref_s:.1f}s on {cores} threads; identical={same}")
    value = statistics.median(times)
    print(json.dumps({
        "metric": "SEISMIC build seconds (fp32, 1M docs)", "value": value, "unit": "s",
        "n_gpus": 1, "steps": len(times), "warmup": 0, "ms_per_step": 1000 * value,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"seismic_build_fp32_{docs.n}_docs", "lambda": 4000, "beta": 400,
                   "alpha": 0.4, "seed": 7},
        "build_s_each": times, "index_sha256": _sha256(ours_path), "reference_gpu_offload": ref,
        "speedup_vs_reference_gpu_offload": None if ref is None else ref["seconds"] / value}))


def serve_sweep(nsparse, idx, docs, qs, cut, hf, rates, seconds=2.0, slots=3):
    """Serving loop under Poisson arrivals: per offered rate, ~`seconds` of
    requests (k 10 or 100 at random, 30% carrying a doc filter that admits a
    random 10% of the docs, labels as random 64-bit external ids); p50/p99
    latency from scheduled arrival to completion, and the completed rate."""
    rng = np.random.default_rng(7)
    srv = nsparse.Server(idx, max_batch=2048, slots=slots)
    srv.set_external_ids(rng.integers(1 << 40, 1 << 62, docs.n, dtype=np.int64))
    bits = np.zeros((docs.n + 64) // 64, dtype=np.uint64)
    ids = rng.choice(docs.n, docs.n // 10, replace=False).astype(np.int64)
    np.bitwise_or.at(bits, ids >> 6, np.left_shift(np.uint64(1), (ids & 63).astype(np.uint64)))
    fid = srv.add_filter(bits)
    # warm-up: every worker's stream and scratch reach their working size
    w = qs.rows(0, min(qs.n, 4000))
    srv.replay(w.indptr, w.indices, w.values, np.where(np.arange(w.n) % 2, 10, 100),
               np.arange(w.n) * 50.0, cut=cut, heap_factor=hf)
    out = []
    for rate in rates:
        before = srv.stats()
        n = int(min(qs.n, max(200, rate * seconds)))
        q = qs.rows(0, n)
        k_per = np.where(rng.random(n) < 0.5, 10, 100).astype(np.int32)
        fper = np.where(rng.random(n) < 0.3, fid, -1).astype(np.int32)
        arrivals = np.cumsum(rng.exponential(1e6 / rate, n))
        t = time.perf_counter()
        _, _, lat = srv.replay(q.indptr, q.indices, q.values, k_per, arrivals, cut=cut,
                               heap_factor=hf, filter_per=fper)
        wall = time.perf_counter() - t
        st = srv.stats()
        lat_ms = np.sort(lat) / 1000.0
        out.append({"offered_qps": rate, "requests": n, "completed_qps": n / wall,
                    "p50_ms": float(np.percentile(lat_ms, 50)),
                    "p99_ms": float(np.percentile(lat_ms, 99)),
                    "mean_batch": (st["requests"] - before["requests"]) /
                                  max(1, st["batches"] - before["batches"])})
        log(json.dumps(out[-1]))
    srv.close()
    return {"cut": cut, "heap_factor": hf, "slots": slots, "max_batch": 2048, "rates": out}


def main():
    global N_DOCS, N_QUERIES, SQ_CUT, SQ_HF
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving sweep")
    ap.add_argument("--cut", type=int, default=None, help="sq8-8.8m: query cut (default 12)")
    ap.add_argument("--heap-factor", type=float, default=None,
                    help="sq8-8.8m: heap factor (default 0.9)")
    ap.add_argument("--serve-slots", default="3",
                    help="serving workers (streams); a comma list runs one sweep per value")
    ap.add_argument("--no-graph", action="store_true",
                    help="time the device-resident step as search_device calls, not graph replays")
    ap.add_argument("--docs", type=int, default=None, help="corpus size (default: the workload's)")
    ap.add_argument("--queries", type=int, default=None, help="queries (default: the workload's)")
    ap.add_argument("--variant", type=int, default=-1, help="search kernel (-1: engine's choice)")
    ap.add_argument("--tuning", type=int, default=0, help="the kernel's tuning value (0: default)")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the device-resident search launches only and exit")
    ap.add_argument("--serve-rates", default="5000,20000,50000,100000,200000",
                    type=lambda s: [float(x) for x in s.split(",") if x],
                    help="offered request rates (queries/s) for the serving sweep")
    ap.add_argument("--digest-out", default="",
                    help="build-1m: write one digest per posting list of the device-built file")
    ap.add_argument("--workload", default="sq8-8.8m",
                    choices=["sq8-8.8m", "fp32-1m", "brutal-100k", "build-1m"],
                    help="sq8-8.8m (default): SEISMIC-SQ at 8.8M docs, the headline; fp32-1m: "
                         "SEISMIC fp32 at 1M docs; brutal-100k: exact brute force; build-1m: "
                         "the device build beside the reference's GPU-offload build")
    args = ap.parse_args()
    if args.workload in ("fp32-1m", "build-1m") and (args.docs or args.queries):
        N_DOCS, N_QUERIES = args.docs or N_DOCS, args.queries or N_QUERIES
        WORKLOAD.update(workload=f"seismic_fp32_{N_DOCS}_docs_{N_QUERIES}_queries", docs=N_DOCS,
                        queries=N_QUERIES)
    SQ_CUT = args.cut if args.cut is not None else SQ_CUT
    SQ_HF = args.heap_factor if args.heap_factor is not None else SQ_HF
    if args.workload == "sq8-8.8m":
        if args.impl == "reference":
            run_reference_sq(args)
        else:
            run_engine_sq(args)
    elif args.workload == "brutal-100k":
        run_engine_brutal(args)
    elif args.workload == "build-1m":
        run_engine_build(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_engine(args)


if __name__ == "__main__":
    main()
