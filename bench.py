#!/usr/bin/env python
"""Benchmark of the casgemm C = A·Aᵀ SpGEMM on B200 (one JSON line on stdout).

Workload (default): the uniform (ER) R-MAT graph of scale 21, edge factor 32
(2,097,152 vertices, 67,108,864 undirected edges, a=b=c=d=0.25, seed 21),
symmetrised, loop- and duplicate-free, values 1.0 (fp64), int32 columns; C =
A·Aᵀ with B = Aᵀ as its own CSR, hybrid accumulator.  The largest
single-matrix configuration that fits one B200 (C alone is about 103 GB).

One step = one full product — the four phases of the reference's drivers
(flop count, symbolic, allocation, numeric) plus freeing C — with A and B
resident in HBM.  `value` = 2 * intermediate products / step time, in
GFLOP/s.  Timed with CUDA events on the launching stream, max over ranks.
The inputs (1.6 GB each) are far larger than the 126 MB L2, so L2 is not
flushed between steps.

`--impl reference` times the reference's own CPU code (built from its sources
into oracle/_ref) on a bounded row sample of the same matrix on the host's
cores.  Under torchrun only rank 0 runs it.

Multi-GPU (torchrun, one rank per GPU): the rows of A are split into
contiguous shards of equal products; each rank computes its shard of C with
B replicated; no data-path collective (scaling: strong, total work fixed).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "contention-aware-spgemm_b200"))

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (family, scale, edge_factor, seed) for R-MAT; the Zipf bipartite
    # join-aggregate stand-in: 850,000 x 2,000,000, 12 M nonzeros, row degrees
    # Zipf(1.2) up to 50,000, column popularity Zipf(1.4) shifted by q_c = 1000
    "er_s21_ef32": ("er", 21, 32, 21),
    "g500_s17_ef8": ("g500", 17, 8, 17),
    "er_s18_ef32": ("er", 18, 32, 18),
    "zipf_850k": ("zipf", 850000, 2000000, 3),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def make_matrix(name):
    """(A, B = A^T): the same CSR for the symmetric R-MAT graphs, the explicit
    transpose for the Zipf bipartite matrix."""
    import casgemm
    fam, s, ef, seed = WORKLOADS[name]
    if fam == "zipf":
        A = casgemm.gen_zipf(s, ef, 50000, 12000000, seed, col_q=1000.0)
        return A, A.transpose()
    A = casgemm.gen_er(s, ef, seed) if fam == "er" else casgemm.gen_g500(s, ef, seed)
    return A, A


def row_products(A, B):
    import casgemm
    return casgemm.row_products_prefix(A, B)


def row_shard(A, B, rank, world, r_end):
    import casgemm
    return casgemm.row_shard(row_products(A, B) if world > 1 else np.zeros(A.num_row + 1, np.int64), rank, world,
                             r_end)


def slice_rows(A, r0, r1):
    import casgemm
    return casgemm.slice_rows(A, r0, r1)


def sample_rows_for(A, B, target_products):
    """Rows [0, R) whose products reach target_products (a bounded CPU sample)."""
    ps = row_products(A, B)
    R = int(np.searchsorted(ps, target_products, side="left"))
    R = max(1, min(R, A.num_row))
    return R, int(ps[R])


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.gpu = str(gpu_index)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", self.gpu], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def gpu_index(local_rank):
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        ids = [x for x in vis.split(",") if x.strip()]
        if local_rank < len(ids):
            return ids[local_rank]
    return local_rank


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_traffic(kernel, workload):
    """Per-launch DRAM traffic of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as fh:
            d = json.load(fh)
        e = d.get(kernel, {}).get(workload)
        return None if e is None else float(e)
    except Exception:
        return None


def cpu_reference(A, B, target_products, steps, warmup):
    """The reference's hybrid driver on rows [0, R): per-step GFLOP/s (its own phase timer).

    Each run is the reference's four phases followed by freeing C, as its
    driver does (src/ams_hybaccspgemm.c:316-343); C is never copied out."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle  # the reference built from its sources (oracle/_ref)
    R, P = sample_rows_for(A, B, target_products)
    As = slice_rows(A, 0, R)
    timer = oracle.RefTimer(As, B, "hybacc", small=False)
    times = []
    for i in range(warmup + steps):
        rt = timer.run()
        if rt is None:
            raise RuntimeError("sample below one morsel")
        if i >= warmup:
            times.append(rt["total_time"])
    t = statistics.mean(times)
    info = oracle.ref_info("hybacc", small=False)
    return {"value": 2.0 * P / t / 1e9, "unit": "GFLOP/s", "cores": info["threads"], "kind": "reference",
            "sample": f"rows [0,{R}) of {A.num_row}: {P} products ({100.0 * P / max(1, total_products(A, B)):.1f}% "
                      f"of the workload), ams_hybaccspgemm kernels, {steps} runs after {warmup} warm-up, "
                      f"mean total_time {t:.3f} s"}


def parity_blocks(A, B, gpu_rows, block_products):
    """Row digests of the GPU product against the reference's own kernels on
    three row blocks (start, middle, end) of about block_products products
    each: the reference runs on A's rows of the block with B whole, its rows
    are sorted and digested in the oracle (cas_csr_digest's row form)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    ps = row_products(A, B)
    total = int(ps[-1])
    m = A.num_row
    blocks = []
    for frac in (0.0, 0.5, 1.0):
        start_p = min(max(0, int(total * frac) - (block_products if frac == 1.0 else 0)), total)
        r0 = int(np.searchsorted(ps, start_p, side="left"))
        r0 = min(r0, m - 1)
        r1 = int(np.searchsorted(ps, int(ps[r0]) + block_products, side="left"))
        r1 = max(r0 + 1, min(r1, m))
        blocks.append((r0, r1))
    out = {"blocks": [], "rows": 0, "match": True, "against": "reference ams_hybaccspgemm kernels (oracle/_ref), "
                                                             "rows sorted, cas_csr_digest row digests"}
    for r0, r1 in blocks:
        res = oracle.ref_row_digests(slice_rows(A, r0, r1), B, "hybacc", small=True)
        ok = res is not None and bool(np.array_equal(res[1], gpu_rows[r0:r1]))
        out["blocks"].append({"rows": [r0, r1], "products": int(ps[r1] - ps[r0]), "match": ok})
        out["rows"] += r1 - r0
        out["match"] = out["match"] and ok
    return out


_TOTAL_P = {}


def total_products(A, B):
    key = id(A)
    if key not in _TOTAL_P:
        import casgemm
        _TOTAL_P[key] = casgemm.intprod(A, B)
    return _TOTAL_P[key]


def run_reference_arm(args, rank, world):
    if rank != 0:
        return 0
    A, B = make_matrix(args.workload)
    base = cpu_reference(A, B, args.ref_products, args.steps, args.warmup)
    line = {"metric": "SpGEMM GFLOP/s (2 x intermediate products / s), C = A*A^T",
            "value": base["value"], "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded R-MAT)", "impl": "reference",
            "config": {"workload": args.workload, "accumulator": "hybacc", "sample": base["sample"]},
            "cpu_baseline": base,
            "e2e": {"value": base["value"], "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_batch_mode(args):
    """The uneven batch: concurrent workers, block-diagonal waves and per-call launches.

    512 G500 R-MAT jobs (scale uniform in 10..17, edge factor in
    {2, 4, 8, 16, 32}, drawn from seed 4), C_j = A_j * A_j^T with int32
    values in 1..8 summed exactly in int64; inputs resident on the device.
    All modes run the same kernels; every job's digest must agree between
    them.  Prints one JSON line (jobs/s of the concurrent mode, with the
    waves and per-call figures and the scale <= 13 subset beside it)."""
    import torch
    import casgemm
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    t0 = time.time()
    spec = casgemm.batch_spec(args.jobs, 4)
    host = [casgemm.batch_job(s, ef, gs) for s, ef, gs in spec]
    log(f"generated {len(host)} jobs in {time.time() - t0:.1f}s")

    def to_dev(M):
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(dev) for x in (M.row_ptrs, M.cols, M.vals)]
        return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, t[0].data_ptr(), t[1].data_ptr(), t[2].data_ptr(),
                                 M.val_type, keep=t)

    jobs = [(to_dev(A), to_dev(B)) for A, B in host]
    small = [i for i, (s, _, _) in enumerate(spec) if s <= 13]
    ctx = casgemm.Context(0)
    for _ in range(args.warmup):
        for mode in ("per_call", "waves", "concurrent"):
            ctx.batch_run([jobs[i] for i in small[:16]], "hybacc", mode)
    torch.cuda.synchronize()
    sampler = ClockSampler(gpu_index(0))
    sampler.start()
    res = {}
    for name, sel in (("all", list(range(len(jobs)))), ("scale_le_13", small)):
        sub = [jobs[i] for i in sel]
        for mode in ("per_call", "waves", "concurrent"):
            secs = []
            for _ in range(args.steps):
                out, st = ctx.batch_run(sub, "hybacc", mode)
                secs.append(st["seconds"])
            res[(name, mode)] = (out, st, statistics.median(secs))
        a = res[(name, "per_call")][0]
        for other in ("waves", "concurrent"):
            b = res[(name, other)][0]
            assert all(x["digest"] == y["digest"] and x["nnz_c"] == y["nnz_c"] for x, y in zip(a, b)), (name, other)
    clocks = sampler.stop()
    # the bound on any batching: every job's own device time, alone (the four
    # phases, CUDA events), summed; batching can only remove what lies
    # between and around those kernels
    alone = []
    for A, B in jobs:
        cc, rt = ctx.spgemm_device(A, B, "hybacc")
        ctx.free(cc)
        alone.append(rt["total_time"])
    alone_s = float(sum(alone))
    heavy = sorted(alone, reverse=True)
    ctx.close()

    def arm(name, mode):
        out, st, sec = res[(name, mode)]
        return {"jobs_per_s": round(len(out) / sec, 3), "seconds": round(sec, 4), "waves": st["waves"],
                "kernel_launches": st["kernel_launches"], "gflops": round(2.0 * st["flop"] / sec / 1e9, 3)}

    all_w, all_p, all_c = arm("all", "waves"), arm("all", "per_call"), arm("all", "concurrent")
    line = {
        "metric": "batched SpGEMM jobs/s (concurrent workers; block-diagonal waves and per-call launches of the "
                  "same kernels beside)",
        "value": all_c["jobs_per_s"], "unit": "jobs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(all_c["seconds"] * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32 in, int64 out", "data": "synthetic (seeded G500 R-MAT)",
        "config": {"workload": f"batch of {len(jobs)} uneven G500 A*A^T jobs (scale 10..17, ef 2..32, seed 4)",
                   "products": res[("all", "waves")][1]["flop"], "nnz_c": res[("all", "waves")][1]["nnz_c"],
                   "inputs": "resident on the device", "digests_agree": True},
        "concurrent": all_c, "waves": all_w, "per_call": all_p,
        "speedup_over_per_call": round(all_c["jobs_per_s"] / all_p["jobs_per_s"], 3),
        "waves_speedup_over_per_call": round(all_w["jobs_per_s"] / all_p["jobs_per_s"], 3),
        "scale_le_13": {"jobs": len(small), "concurrent": arm("scale_le_13", "concurrent"),
                        "waves": arm("scale_le_13", "waves"), "per_call": arm("scale_le_13", "per_call"),
                        "speedup_over_per_call": round(arm("scale_le_13", "concurrent")["jobs_per_s"]
                                                       / arm("scale_le_13", "per_call")["jobs_per_s"], 3)},
        "gpu_launches": all_c["kernel_launches"],
        "clocks": clocks,
        "bound": {"alone_device_seconds": round(alone_s, 4),
                  "jobs_per_s_if_no_overhead": round(len(jobs) / alone_s, 3),
                  "max_speedup_over_per_call": round(all_p["seconds"] / alone_s, 3),
                  "heaviest_8_jobs_share": round(sum(heavy[:8]) / alone_s, 3),
                  "how": "sum over jobs of each job's four phases alone (CUDA events); serial batching can "
                         "only remove the host waits and launches between them, while concurrent jobs can also "
                         "share the SMs a small job leaves idle"},
    }
    print(json.dumps(line), flush=True)
    return 0


def serve_pool(n_pool, seed):
    """Distinct requests of the serving stream: half G500 R-MAT (scale
    uniform in [12, 19], edge factor uniform in 4..32), half Zipf bipartite
    (rows log-uniform in [10k, 500k], 2.35 columns per row as in the 850k x
    2M join-aggregate set, row law Zipf(1.2) with the largest row scaled
    from 50,000 at 850k rows, column law Zipf(1.4) shifted by q_c = 1000,
    average degree uniform in [8, 24]); values 1.0."""
    import casgemm
    rng = np.random.default_rng(seed)
    pool = []
    for i in range(n_pool):
        if i % 2 == 0:
            s = int(round(rng.uniform(12, 19)))
            ef = int(rng.integers(4, 33))
            A = casgemm.gen_g500(s, ef, int(rng.integers(1 << 31)))
            name = f"g500_s{s}_ef{ef}"
        else:
            nr = int(round(np.exp(rng.uniform(np.log(1e4), np.log(5e5)))))
            nc = int(2.35 * nr)
            deg = float(rng.uniform(8, 24))
            amax = int(min(nc, max(deg * 4, 50000 * nr / 850000)))
            A = casgemm.gen_zipf(nr, nc, amax, int(deg * nr), int(rng.integers(1 << 31)), col_q=1000.0)
            name = f"zipf_{nr}x{nc}_d{deg:.0f}"
        pool.append((name, A, A.transpose()))
    return pool


def run_serve_mode(args):
    """Serving stream: Poisson arrivals at --rate requests/s, requests drawn
    from a pool of distinct matrices, admitted by the 60 GB bound; p50/p99
    latency (completion - arrival) and jobs/s.  Every result's digest must
    equal the digest of the same request run alone."""
    import threading
    import casgemm
    t0 = time.time()
    pool = serve_pool(args.pool, 5)
    log(f"generated a pool of {len(pool)} requests in {time.time() - t0:.1f}s")
    if not args.host_operands:
        # operands resident on the device: each distinct matrix uploaded once
        import torch
        torch.cuda.set_device(0)
        pool = [(name, casgemm.DeviceCsr.upload(A), casgemm.DeviceCsr.upload(B)) for name, A, B in pool]
        torch.cuda.synchronize()
    # alone: each distinct request by itself on a one-slot server
    solo = {}
    with casgemm.Server(slots=1) as srv:
        for k, (name, A, B) in enumerate(pool):
            r = srv.wait(srv.submit(A, B))
            if r["status"] != 0:
                raise RuntimeError(f"{name}: status {r['status']}")
            solo[k] = (r["digest"], r["nnz_c"], r["flop"], r["t_done"] - r["t_admit"])
    rng = np.random.default_rng(55)
    picks = rng.integers(0, len(pool), args.requests)
    gaps = rng.exponential(1.0 / args.rate, args.requests)
    sampler = ClockSampler(gpu_index(0))
    sampler.start()
    ids = [None] * args.requests
    with casgemm.Server(slots=args.slots, mem_budget=60e9) as srv:
        start = srv.clock()

        def feeder():
            t = start
            for i in range(args.requests):
                t += gaps[i]
                d = t - srv.clock()
                if d > 0:
                    time.sleep(d)
                _, A, B = pool[picks[i]]
                ids[i] = srv.submit(A, B)

        th = threading.Thread(target=feeder)
        th.start()
        th.join()
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    clocks = sampler.stop()
    bad = [i for i, r in enumerate(res) if r["status"] != 0 or (r["digest"], r["nnz_c"]) != solo[picks[i]][:2]]
    if bad:
        raise RuntimeError(f"{len(bad)} results differ from the same request alone (first: {bad[0]})")
    lat = np.array([r["t_done"] - r["t_submit"] for r in res])
    span = max(r["t_done"] for r in res) - min(r["t_submit"] for r in res)
    flop = sum(r["flop"] for r in res)
    line = {
        "metric": "SpGEMM serving: jobs/s with p50/p99 latency (continuous batching, 60 GB admission budget)",
        "value": round(args.requests / span, 3), "unit": "jobs/s", "n_gpus": 1, "steps": args.requests,
        "warmup": len(pool), "ms_per_step": round(1e3 * span / args.requests, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded G500 R-MAT and Zipf)",
        "config": {"workload": f"{args.requests} requests, Poisson {args.rate}/s, pool of {len(pool)} distinct",
                   "slots": args.slots, "budget_bytes": 60e9, "products": flop,
                   "operands": "host, copied per request" if args.host_operands else
                   "resident on the device (each distinct matrix uploaded once before the stream)"},
        "latency_s": {"p50": round(float(np.percentile(lat, 50)), 4), "p99": round(float(np.percentile(lat, 99)), 4),
                      "max": round(float(lat.max()), 4)},
        "gflops": round(2.0 * flop / span / 1e9, 3),
        "server": st, "chunked_requests": int(st["chunked"]), "rejected": int(st["failed"]),
        "alone_service_s": {"p50": round(float(np.percentile([v[3] for v in solo.values()], 50)), 4),
                            "max": round(float(max(v[3] for v in solo.values())), 4)},
        "results_equal_alone": True,
        "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--mode", default="product", choices=["product", "batch", "serve"],
                    help="product: one large SpGEMM (the headline); batch: the uneven batch of jobs; "
                         "serve: the Poisson request stream")
    ap.add_argument("--requests", type=int, default=200, help="serve mode: requests in the stream")
    ap.add_argument("--rate", type=float, default=5.0, help="serve mode: Poisson arrival rate, requests/s")
    ap.add_argument("--slots", type=int, default=4, help="serve mode: requests in flight at once")
    ap.add_argument("--pool", type=int, default=32, help="serve mode: distinct requests the stream draws from")
    ap.add_argument("--host-operands", action="store_true",
                    help="serve mode: submit host operands (copied per request) instead of resident ones")
    ap.add_argument("--jobs", type=int, default=512, help="batch mode: number of jobs")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="cas", choices=["cas", "reference"])
    ap.add_argument("--workload", default="er_s21_ef32", choices=sorted(WORKLOADS))
    ap.add_argument("--accum", default="hybacc", choices=["hash", "hsersc", "hybacc"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--parity-products", type=float, default=3e7,
                    help="products in each of the three row blocks checked against the reference")
    ap.add_argument("--ref-products", type=float, default=4e8,
                    help="products in the CPU reference's row sample")
    ap.add_argument("--row-fraction", type=float, default=1.0,
                    help="use only the first fraction of A's rows (profiling captures; B stays whole)")
    ap.add_argument("--tune", default=None, metavar="CACHE.json",
                    help="pick the row routing with casgemm.Autotuner (cached in CACHE.json) before timing")
    ap.add_argument("--esc-form", type=int, default=None, choices=[0, 1, 2],
                    help="bucketed ESC kernel form (cas_tuning.esc_form); default: the library's")
    ap.add_argument("--out-blocks", type=int, default=None,
                    help="row blocks of the e2e leg's host C (cas_tuning.out_blocks; 0 by size, 1 one block)")
    ap.add_argument("--bin-order", type=int, default=None, choices=[0, 1],
                    help="numeric bins interleaved (0) or grouped (1) on the streams (cas_tuning.bin_order)")
    ap.add_argument("--heavy-split", type=int, default=None, choices=[0, 1],
                    help="split the heaviest dense rows across blocks (cas_tuning.heavy_split); default: the library's")
    ap.add_argument("--assemble", action="store_true",
                    help="N > 1: assemble C's row shards on rank 0 after the timed steps (reported, not timed)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    if args.mode == "batch":
        return run_batch_mode(args) if rank == 0 else 0
    if args.mode == "serve":
        return run_serve_mode(args) if rank == 0 else 0

    import torch
    import casgemm
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())

    t0 = time.time()
    A, B = make_matrix(args.workload)
    r_end = max(1, int(round(A.num_row * args.row_fraction)))
    r0, r1 = row_shard(A, B, rank, world, r_end)
    As = slice_rows(A, r0, r1)
    log(f"[rank {rank}] matrix {args.workload}: n={A.num_row} nnz={A.nnz} rows [{r0},{r1}) in {time.time() - t0:.1f}s")

    def to_dev(M):
        rp = torch.from_numpy(np.ascontiguousarray(M.row_ptrs)).to(dev)
        c = torch.from_numpy(np.ascontiguousarray(M.cols)).to(dev)
        v = torch.from_numpy(np.ascontiguousarray(M.vals)).to(dev)
        return casgemm.DeviceCsr(M.num_row, M.num_col, M.nnz, rp.data_ptr(), c.data_ptr(), v.data_ptr(),
                                 keep=(rp, c, v))

    dA, dB = to_dev(As), to_dev(B)
    ctx = casgemm.Context(dev.index)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)

    tuning = None
    if args.esc_form is not None:
        ctx.set_tuning(esc_form=args.esc_form)
    if args.heavy_split is not None:
        ctx.set_tuning(heavy_split=args.heavy_split)
    if args.bin_order is not None:
        ctx.set_tuning(bin_order=args.bin_order)
    if args.out_blocks is not None:
        ctx.set_tuning(out_blocks=args.out_blocks)
    if args.tune:
        tuner = casgemm.Autotuner(ctx, args.tune)
        key = casgemm.Autotuner.key(As, B)
        tuning = dict(tuner.tune(key, dA, dB, args.accum), key=key)
        tuner.apply(key)
        log(f"[rank {rank}] tuning {tuning}")

    def step():
        cc, rt = ctx.spgemm_device(dA, dB, args.accum)
        ctx.free(cc)
        return rt

    for _ in range(args.warmup):
        step()
    st_w = ctx.stats()
    launches0 = st_w["kernel_launches"]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    sampler = ClockSampler(gpu_index(local_rank))
    sampler.start()
    time.sleep(0.3)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    rts = []
    for _ in range(args.steps):
        rts.append(step())
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop()
    if dist:
        dist.barrier()
    stats = ctx.stats()
    launches = stats["kernel_launches"] - launches0
    elapsed_ms = ev0.elapsed_time(ev1)
    P_local = stats["flop"]
    nnz_local = stats["nnz_c"]
    if dist:
        t = torch.tensor([elapsed_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms = float(t.item())
        tot = torch.tensor([P_local, nnz_local, launches], device=dev, dtype=torch.float64)
        dist.all_reduce(tot)
        P_total, nnz_total, launches_total = int(tot[0].item()), int(tot[1].item()), int(tot[2].item())
    else:
        P_total, nnz_total, launches_total = P_local, nnz_local, launches
    ms_step = elapsed_ms / args.steps
    value = 2.0 * P_total / (ms_step * 1e-3) / 1e9

    # row digests of one product for the parity check against the reference
    cc, _ = ctx.spgemm_device(dA, dB, args.accum)
    _, gpu_rows = ctx.digest(cc, rows=True)
    assembly = None
    if dist and args.assemble:
        # C's row shards assembled on rank 0 (all-gather of the shard sizes,
        # then point-to-point NCCL transfers), timed on the device, max over
        # ranks; rank 0 checks the assembled rows' digests against the shards'
        rp_t, col_t, val_t = casgemm.device_tensors(cc)
        torch.cuda.synchronize()
        dist.barrier()
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ea.record()
        got = casgemm.gather_shards(rp_t, col_t, val_t, r0, r1, r_end)
        eb.record()
        torch.cuda.synchronize()
        t = torch.tensor([ea.elapsed_time(eb)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        shard_rows = [None] * world
        dist.all_gather_object(shard_rows, gpu_rows)
        if rank == 0:
            full = casgemm.CasCsr(r_end, B.num_col, int(got[0][-1]), got[0].data_ptr(),
                                  got[1].data_ptr(), got[2].data_ptr(), 4, 0, 1, 0)
            _, rows_full = ctx.digest(full, rows=True)
            match = bool(np.array_equal(rows_full, np.concatenate(shard_rows)))
            assembly = {"ms": round(float(t.item()), 3), "nnz": int(got[0][-1]),
                        "bytes": 8.0 * (r_end + 1) + 12.0 * float(got[0][-1]), "row_digests_match": match,
                        "how": "all-gather of shard sizes, point-to-point NCCL sends of columns, values and "
                               "row pointers to rank 0"}
        del got, rp_t, col_t, val_t
    ctx.free(cc)

    # per-kernel times for the roofline: extra steps with the bins run one at
    # a time and each bin kernel timed by CUDA events on its stream
    ctx.set_profiling(True)
    bin_ms, bin_bytes, bin_nnz = {}, {}, {}
    n_prof = 2
    ovf_rows, ovf_ms = 0, 0.0
    for _ in range(n_prof):
        step()
        s = ctx.stats()
        for k, v in s["numc_bin_ms"].items():
            bin_ms[k] = bin_ms.get(k, 0.0) + v / n_prof
            bin_bytes[k] = bin_bytes.get(k, 0.0) + s["numc_bin_bytes"][k] / n_prof
            bin_nnz[k] = s["numc_bin_nnz"][k]
        ovf_rows, ovf_ms = s["esc_overflow_rows"], ovf_ms + s["esc_overflow_ms"] / n_prof
        if s["fused_rows"]:
            bin_ms["fused"] = bin_ms.get("fused", 0.0) + s["fused_ms"] / n_prof
            bin_bytes["fused"] = bin_bytes.get("fused", 0.0) + s["fused_bytes"] / n_prof
    ctx.set_profiling(False)

    # roofline of the dominant kernel (the numeric bin with the most device time)
    peak, peak_kind = measured_peak()
    dom = max(bin_ms, key=lambda k: bin_ms[k])
    dom_ms = bin_ms[dom]
    dom_bytes = bin_bytes[dom]
    achieved = dom_bytes / (dom_ms * 1e-3) / 1e9 if dom_ms > 0 else 0.0
    kernel_name = {"tiny": "k_numc_tiny<256>", "hash256": "k_numc_hash<256,9>", "hash1k": "k_numc_hash<256,11>",
                   "hash4k": "k_numc_hash<512,13>", "dense": "k_numc_dense<512>"}.get(dom)
    # the index form runs the fused rows and the ESC bins over 4096 products when esc_form is 1
    form = ctx.get_tuning().get("esc_form", 1)
    idx_form = form >= 1
    if dom == "fused":
        kernel_name = "k_numc_esc_%s<256,5120,11,fused%s>" % ("idx" if idx_form else "msd",
                                                            ",keys in registers" if form == 2 else "")
    if kernel_name is None and dom.startswith("esc"):
        shape = {"esc1k": "1024,9", "esc2k": "2048,9", "esc3k": "3072,10", "esc4k": "4096,10",
                 "esc5k": "4800,11", "esc6k": "6144,11", "esc8k": "8192,11"}[dom]
        big = dom in ("esc5k", "esc6k", "esc8k")
        kernel_name = "k_numc_esc_%s<256,%s%s>" % ("idx" if idx_form and big else "msd", shape,
                                                  ",keys in registers" if form == 2 and dom in ("esc5k", "esc6k")
                                                  else "")
    alg_bytes_total = 12.0 * (A.nnz if world == 1 else As.nnz) + 12.0 * P_local + 12.0 * nnz_local + 16.0 * (As.num_row + 1)
    pipe_frac = alg_bytes_total / (ms_step * 1e-3) / (peak * 1e9)

    line = {
        "metric": "SpGEMM GFLOP/s (2 x intermediate products / s), C = A*A^T",
        "value": round(value, 3), "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms_step, 3), "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded R-MAT, values 1.0)",
        "config": {"workload": args.workload, "accumulator": args.accum, "row_fraction": args.row_fraction,
                   "products": P_total, "nnz_c": nnz_total, "nnz_a": A.nnz, "n": A.num_row,
                   "l2": f"not flushed: inputs ({12 * A.nnz / 1e9:.2f} GB each) exceed the 126 MB L2",
                   "parallelism": f"row shards x{world}" if world > 1 else "1 GPU",
                   "phases_ms_last_step": {k: round(v * 1e3, 3) for k, v in rts[-1].items()},
                   "tuning": tuning if tuning else ctx.get_tuning()},
        "roofline": {"bound": "hbm", "kernel": kernel_name, "bin": dom,
                     "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                     "alg_bytes_per_launch": dom_bytes, "launch_ms": round(dom_ms, 3),
                     "timing": "CUDA events around the kernel, bins serialised, mean of 2 extra steps",
                     "traffic": committed_traffic(kernel_name, args.workload)},
        "numc_bins_ms": {k: round(v, 3) for k, v in bin_ms.items() if v > 0},
        "numc_bins_nnz": {k: int(v) for k, v in bin_nnz.items() if v > 0},
        "esc_radix_fallback": {"rows": ovf_rows, "ms": round(ovf_ms, 3)},
        "pipeline_roofline": {"alg_bytes": alg_bytes_total, "frac": round(pipe_frac, 4),
                              "formula": "12*nnz(A)+12*P+12*nnz(C)+16*(m+1) over the step time"},
        "gpu_launches": launches_total,
        "clocks": clocks,
    }
    if assembly is not None:
        line["assembly"] = assembly

    # end to end through the public C ABI with pinned host buffers: H2D of A and
    # B, the product, D2H of C into host memory, every step
    if not args.no_e2e:
        pin = lambda x: torch.from_numpy(np.ascontiguousarray(x)).pin_memory()  # noqa: E731
        hA = [pin(As.row_ptrs), pin(As.cols), pin(As.vals)]
        hB = hA if (world == 1 and B is A) else [pin(B.row_ptrs), pin(B.cols), pin(B.vals)]
        ca = casgemm.CasCsr(As.num_row, As.num_col, As.nnz, hA[0].data_ptr(), hA[1].data_ptr(), hA[2].data_ptr(),
                            4, 0, 0, 0)
        cb = casgemm.CasCsr(B.num_row, B.num_col, B.nnz, hB[0].data_ptr(), hB[1].data_ptr(), hB[2].data_ptr(),
                            4, 0, 0, 0)
        import ctypes
        walls, h2d, d2h = [], 0.0, 0.0
        for it in range(1 + args.e2e_steps):  # one untimed warm-up call first
            cc = casgemm.CasCsr()
            cc.on_device, cc.col_bytes = 0, 4
            torch.cuda.synchronize()
            if dist:
                dist.barrier()
            tw = time.perf_counter()
            stt = ctx.lib.cas_spgemm(ctx.h, casgemm.ACCUM[args.accum], ctypes.byref(ca), ctypes.byref(cb),
                                     ctypes.byref(cc), None)
            if stt != 0:
                raise casgemm.CasError(stt, ctx.lib.cas_last_error(ctx.h).decode())
            _ = int(np.ctypeslib.as_array(ctypes.cast(cc.row_ptrs, ctypes.POINTER(ctypes.c_int64)), (cc.num_row + 1,))[-1])
            if it > 0:
                walls.append(time.perf_counter() - tw)
            s = ctx.stats()
            h2d, d2h, d2h_direct = s["h2d_bytes"], s["d2h_bytes"], s["d2h_direct_bytes"]
            out_blocks = s["out_blocks"]
            ctx.lib.cas_csr_free(ctx.h, ctypes.byref(cc))
        wall = statistics.mean(walls)
        if dist:
            t = torch.tensor([wall], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            wall = float(t.item())
        line["e2e"] = {"value": round(2.0 * P_total / wall / 1e9, 3), "unit": "GFLOP/s",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "steps": args.e2e_steps, "s_per_step": round(wall, 3),
                       "warmup": 1, "d2h_direct_bytes_per_step": d2h_direct, "out_blocks": out_blocks,
                       "path": "cas_spgemm on pinned host A, B; C returned in host memory (after one untimed "
                               "call, so C's host blocks are the context's resident ones, registered with "
                               "CUDA when they came back; d2h_direct bytes went to them by DMA directly), "
                               "computed in out_blocks row blocks, each copied out while the next is computed"}
        del hA, hB

    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        dA = dB = None
        torch.cuda.empty_cache()
        try:
            line["cpu_baseline"] = cpu_reference(A, B, args.ref_products, steps=3, warmup=1)
        except Exception as e:  # reported, not fatal
            line["cpu_baseline"] = {"value": None, "error": str(e)}
        if args.row_fraction == 1.0:
            try:
                line["parity"] = parity_blocks(A, B, gpu_rows, int(args.parity_products))
            except Exception as e:  # reported, not fatal
                line["parity"] = {"match": None, "error": str(e)}
    ctx.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
