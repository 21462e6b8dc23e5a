#!/usr/bin/env python
"""Benchmark of the B200 quantized-graph query path (one JSON line on stdout).

Workload (default, "batched-1m128"): N = 1,000,000 base vectors, D = 128,
float32 integers from a seeded Gaussian mixture of 1,024 isotropic clusters
(centres uniform in [0, 255], sigma 20, clipped to [0, 255], rounded);
degree_bound 32, build EF 400, 3 build rounds; 10,000 queries from the same
mixture; k = 10; ef = the smallest of {64, 128, 256} whose best-10-of-pool
recall@10 against an FP64 brute-force ground truth is >= 0.95. Synthetic data
stands in for the reference's datasets (none ship with it).

One "step" = one batched search of all 10,000 queries (the work-order kernel
and sort, one persistent launch of the search kernel the autotuner picks, on
this workload the batch kernel with the lazy search heap, and the exact kernel
over the queries that outgrew its capacities, usually none), inputs resident
in HBM. The L2 is flushed between steps (a 256 MiB write), outside the timed
events. `e2e` times the same step through the host-buffer C-ABI call
(lqg_search_batch): pinned host queries in, ids out, inside the timed region.

The index is built on the GPU by the package's builder (the reference's own
builder yields graphs whose recall stays far below 0.95) and cached under
$LQG_BENCH_CACHE (default /tmp/lqg_bench) together with the ground truth, so
the reference arm and this arm search the same index file.

--impl reference: the reference's own CPU search (QuantizedGraph::search,
compiled from its sources into oracle/_ref by oracle/Makefile; the C oracle
port if that is absent) on all host cores, same index file, same ef and k,
each step a bounded sample of the queries.

Multi-GPU (torchrun, N > 1): replicas only. Every rank holds the same index
and searches its own 10,000 queries (seeded by rank); no collective on the
data path; value = all queries / max-over-ranks time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import ctypes as C
import hashlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "QPS @ recall@10≥0.95: batched vs plain GPU vs CPU; p50/p99 ms; HBM GB/s"
BUILDER_VERSION = "gpu-builder-5"

WORKLOADS = {
    "batched-1m128": dict(n=1_000_000, dim=128, gen="int_mixture", clusters=1024, lo=0.0,
                          hi=255.0, sigma=20.0, deg=32, efb=400, iters=3, random_edges=8,
                          path_take=64, far_budget=8, nq=10_000, k=10, efs=(64, 128, 256),
                          k_extra=100),
    "small-100k64": dict(n=100_000, dim=64, gen="uniform", deg=32, efb=200, iters=3,
                         random_edges=4, path_take=64, far_budget=4, nq=1000, k=10,
                         efs=(20, 40, 60, 100, 200), k_extra=100, knn_compare=True),
    # Uneven batch, high dimension (per-query ef and k;
    # CUDA-graph replay timed beside the eager launch)
    "uneven-1m960": dict(n=1_000_000, dim=960, gen="gauss_mixture", clusters=256, sigma=0.3,
                         deg=64, efb=400, iters=3, random_edges=8, path_take=64, far_budget=8,
                         nq=4096, kind="uneven", ef_choices=(32, 64, 128, 256, 512),
                         k_choices=(1, 10, 100)),
    # Index build with BF16 tensor-core pruning against the
    # FP32 prune (unit-length rows; centre entries N(0, 1), sigma 0.3)
    "build-1m768": dict(n=1_000_000, dim=768, gen="gauss_mixture_unit", clusters=2048, sigma=0.3,
                        deg=64, efb=400, iters=3, random_edges=8, path_take=64, far_budget=8,
                        nq=2000, kind="build", ef=128),
    # the build workload's data at N = 100,000: a build small enough to profile
    "build-100k768": dict(n=100_000, dim=768, gen="gauss_mixture_unit", clusters=2048, sigma=0.3,
                          deg=64, efb=400, iters=3, random_edges=8, path_take=64, far_budget=8,
                          nq=2000, kind="build", ef=128),
    # Serving loop, open-loop Poisson arrivals (4 s of
    # arrivals at every rate: 2M distinct queries cover 500 k/s)
    "serving-10m96": dict(n=10_000_000, dim=96, gen="gauss_mixture", clusters=4096, sigma=0.25,
                          deg=32, efb=300, iters=3, random_edges=8, path_take=64, far_budget=8,
                          nq=2_000_000, kind="serving", rates=(20_000, 100_000, 500_000),
                          k_choices=(10, 100), ef_choices=(50, 100, 200, 500), seconds=4.0),
}


# a launch shape per kernel mode for --mode: (mode, lanes_per_cand,
# visited_bits, warps_per_block, heap_warps, heap_scap)
FIXED_TUNING = {1: (1, 4, 10, 8, 4, 1024), 2: (2, 4, 10, 8, 4, 1024), 3: (3, 4, 10, 8, 4, 512),
                4: (4, 4, 10, 8, 4, 256), 5: (5, 2, 10, 8, 4, 256), 6: (6, 2, 10, 8, 4, 256)}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ---------------------------------------------------------------- data
def gen_data(w, which: str, rank: int = 0):
    """Base vectors (seed 0) or queries (seed 1, +rank for replicas)."""
    n = w["n"] if which == "base" else w["nq"]
    if w["gen"] == "uniform":
        rng = np.random.default_rng(0 if which == "base" else 1 + 1000 * rank)
        return rng.random((n, w["dim"]), dtype=np.float32)
    if w["gen"] in ("gauss_mixture", "gauss_mixture_unit"):
        # centre entries N(0, 1), isotropic sigma, float; "_unit": rows scaled
        # to unit L2 norm
        centres = np.random.default_rng(0).normal(0.0, 1.0, (w["clusters"], w["dim"]))
        rng = np.random.default_rng(100 if which == "base" else 1 + 1000 * rank)
        out = np.empty((n, w["dim"]), dtype=np.float32)
        step = 1 << 17
        for s in range(0, n, step):
            m = min(step, n - s)
            lab = rng.integers(0, w["clusters"], m)
            x = centres[lab] + rng.normal(0.0, w["sigma"], (m, w["dim"]))
            if w["gen"] == "gauss_mixture_unit":
                x /= np.linalg.norm(x, axis=1, keepdims=True)
            out[s:s + m] = x
        return out
    centres = np.random.default_rng(0).uniform(w["lo"], w["hi"], (w["clusters"], w["dim"]))
    rng = np.random.default_rng(100 if which == "base" else 1 + 1000 * rank)
    out = np.empty((n, w["dim"]), dtype=np.float32)
    step = 1 << 17
    for s in range(0, n, step):
        m = min(step, n - s)
        lab = rng.integers(0, w["clusters"], m)
        x = centres[lab] + rng.normal(0.0, w["sigma"], (m, w["dim"]))
        out[s:s + m] = np.clip(np.rint(x), w["lo"], w["hi"])
    return out


def cache_dir():
    d = os.environ.get("LQG_BENCH_CACHE", "/tmp/lqg_bench")
    os.makedirs(d, exist_ok=True)
    return d


def key_of(name, w):
    h = hashlib.sha1(json.dumps([name, sorted(w.items()), BUILDER_VERSION], default=str).encode())
    return f"{name}-{h.hexdigest()[:10]}"


def index_path(name, w):
    return os.path.join(cache_dir(), key_of(name, w) + ".idx")


def gt_path(name, w, rank, nq):
    return os.path.join(cache_dir(), key_of(name, w) + f".gt{rank}-{nq}.npy")


def workload_str(name, w, nq, k, ef):
    """The `config.workload` string; both arms print the same one."""
    return (f"{name}: N={w['n']} D={w['dim']} deg={w['deg']} EF={w['efb']} "
            f"(random_edges={w['random_edges']}, path_take={w['path_take']}, "
            f"far_budget={w['far_budget']}), {nq} queries/GPU, k={k}, ef={ef}")


# ------------------------------------------------- the prebuilt bench graph
# The reference arm runs first on a fresh machine and must neither touch the
# GPU nor load this package's library, yet it has to search the same index
# file as the GPU arm. So the GPU builder's graph for the default workload is
# carried with the repository copy (bench_data/, not committed: neighbour ids
# packed at ceil(log2 N) bits, the entry point, the FP64 ground truth of the
# rank-0 queries and the SHA-256 of the whole index file). On the CPU the arm
# regenerates the base vectors from their seed, SQ8-encodes them with the
# reference's own encoder (oracle/_ref), writes the reference's file layout
# and checks the hash; only when that is impossible does it fall back to a
# child process that runs the GPU builder (recorded in its line).
DATA_DIR = os.path.join(ROOT, "bench_data")


def _id_bits(n):
    """Bits per packed id: ceil(log2 n) rounded up to a multiple of 4."""
    return max(4, -(-int(n - 1).bit_length() // 4) * 4)


def _pack_ids(ids, bits):
    """u32 ids < 2^bits -> bytes: two ids per 2*bits/8 bytes, little-endian."""
    v = np.ascontiguousarray(ids, dtype=np.uint64).reshape(-1)
    if len(v) % 2:
        v = np.concatenate([v, np.zeros(1, np.uint64)])
    word = v[0::2] | (v[1::2] << np.uint64(bits))
    nb = 2 * bits // 8
    return word.view(np.uint8).reshape(-1, 8)[:, :nb].tobytes()


def _unpack_ids(buf, bits, count):
    nb = 2 * bits // 8
    a = np.zeros((len(buf) // nb, 8), np.uint8)
    a[:, :nb] = np.frombuffer(buf, np.uint8).reshape(-1, nb)
    word = a.view(np.uint64).reshape(-1)
    mask = np.uint64((1 << bits) - 1)
    out = np.empty((len(word), 2), np.uint64)
    out[:, 0] = word & mask
    out[:, 1] = (word >> np.uint64(bits)) & mask
    return out.reshape(-1)[:count].astype(np.uint32)


def _sha256(path):
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for blk in iter(lambda: f.read(1 << 24), b""):
            h.update(blk)
    return h.hexdigest()


def export_shipped(name, w, part, nparts, outdir):
    """Writes part `part` of `nparts` of the cached index's neighbour lists
    (packed), plus the metadata and (part 0) the rank-0 ground truth, under
    outdir; the cached index and ground truth must exist (a GPU-arm run)."""
    from oracle.oracle import read_index

    path = index_path(name, w)
    arr = read_index(path, w["n"], w["dim"], w["deg"])
    bits = _id_bits(w["n"])
    rows = np.array_split(np.arange(w["n"]), nparts)[part]
    key = key_of(name, w)
    os.makedirs(outdir, exist_ok=True)
    with open(os.path.join(outdir, f"{key}.nbrs{part}of{nparts}.bin"), "wb") as f:
        f.write(_pack_ids(arr.nbrs[rows[0]:rows[-1] + 1], bits))
    meta = {"workload": name, "key": key, "n": w["n"], "dim": w["dim"], "deg": w["deg"],
            "entry": arr.entry, "bits": bits, "nparts": nparts,
            "sha256": _sha256(path), "builder": BUILDER_VERSION}
    with open(os.path.join(outdir, f"{key}.meta{part}.json"), "w") as f:
        json.dump(meta, f)
    if part == 0:
        gt = np.load(gt_path(name, w, 0, w["nq"]))
        np.savez_compressed(os.path.join(outdir, f"{key}.gt0.npz"), gt=gt.astype(np.int32))
    print(json.dumps(meta), flush=True)


def assemble_shipped(name, w, base):
    """CPU only: the cached index file (and rank-0 ground truth) from
    bench_data/ and the regenerated base vectors. Returns a note for the
    JSON line, or None when bench_data/ has no complete, matching copy."""
    from oracle.oracle import IndexArrays, RefHarness, ref_available, sq8_quantize, write_index

    key = key_of(name, w)
    try:
        with open(os.path.join(DATA_DIR, f"{key}.meta0.json")) as f:
            meta = json.load(f)
        nparts = meta["nparts"]
        metas = [meta]
        for p in range(1, nparts):
            with open(os.path.join(DATA_DIR, f"{key}.meta{p}.json")) as f:
                metas.append(json.load(f))
    except (OSError, ValueError, KeyError):
        return None
    if any(m["sha256"] != meta["sha256"] for m in metas):
        return None
    rows = np.array_split(np.arange(w["n"]), nparts)
    nb = np.empty((w["n"], w["deg"]), np.uint32)
    for p in range(nparts):
        try:
            with open(os.path.join(DATA_DIR, f"{key}.nbrs{p}of{nparts}.bin"), "rb") as f:
                buf = f.read()
        except OSError:
            return None
        cnt = len(rows[p]) * w["deg"]
        nb[rows[p][0]:rows[p][-1] + 1] = _unpack_ids(buf, meta["bits"], cnt).reshape(-1, w["deg"])
    if ref_available():
        codes, params = RefHarness().sq8_quantize(base)
        enc = "the reference's sq8_quantize (oracle/_ref)"
    else:
        codes, params = sq8_quantize(base)
        enc = "the oracle's SQ8 encoder"
    path = index_path(name, w)
    tmp = path + f".tmp{os.getpid()}"
    write_index(tmp, IndexArrays(w["n"], w["dim"], w["deg"], meta["entry"], base, nb, codes, params))
    if _sha256(tmp) != meta["sha256"]:
        os.remove(tmp)
        return None
    os.replace(tmp, path)
    gt = np.load(os.path.join(DATA_DIR, f"{key}.gt0.npz"))["gt"].astype(np.int64)
    np.save(gt_path(name, w, 0, len(gt)), gt)
    return (f"index file assembled on the CPU from bench_data/ (GPU builder's graph, "
            f"{meta['builder']}) with codes from {enc}; SHA-256 matches the built file")


def prepare_in_child(name, w):
    """Fallback of the reference arm: the GPU builder and the GPU ground truth
    run in a child process, so this process loads neither."""
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--prepare",
                        "--workload", name], stdout=subprocess.PIPE, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"--prepare failed with {r.returncode}")
    return "index file built and ground truth computed by a child process (GPU builder)"


def get_index_file(name, w, base, device):
    """Builds (GPU builder) or reuses the cached index file."""
    import liteqg_b200

    path = index_path(name, w)
    if os.path.exists(path):
        return path, 0.0
    if assemble_shipped(name, w, base) is not None:
        return path, 0.0
    ix = liteqg_b200.Index("QG", "L2", w["n"], w["dim"], w["deg"], device=device)
    t = time.perf_counter()
    ix.build_index(base, w["efb"], num_iter=w["iters"], random_edges=w["random_edges"],
                   path_take=w["path_take"], far_budget=w["far_budget"])
    tb = time.perf_counter() - t
    tmp = path + f".tmp{os.getpid()}"
    ix.save(tmp)
    os.replace(tmp, path)
    ix.close()
    return path, tb


def ground_truth(name, w, base, queries, device, rank):
    """FP64 brute-force top-100 ids per query (GPU, chunked), cached."""
    import torch

    path = gt_path(name, w, rank, len(queries))
    if os.path.exists(path):
        return np.load(path)
    dev = torch.device("cuda", device)
    xb = torch.from_numpy(base).to(dev, torch.float64)
    nb = (xb * xb).sum(1)
    kk = 100
    out = np.empty((len(queries), kk), np.int64)
    qc = max(16, min(1024, (4 << 30) // (8 * len(base))))  # distance block <= 4 GiB
    for s in range(0, len(queries), qc):
        q = torch.from_numpy(queries[s:s + qc]).to(dev, torch.float64)
        d = nb[None, :] - 2.0 * (q @ xb.T) + (q * q).sum(1)[:, None]
        out[s:s + len(q)] = torch.topk(d, kk, dim=1, largest=False).indices.cpu().numpy()
    del xb
    torch.cuda.empty_cache()
    np.save(path, out)
    return out


def recall_at(pool_ids, gt, k):
    hits = 0
    for i in range(len(gt)):
        hits += len(set(pool_ids[i, :k].tolist()) & set(gt[i, :k].tolist()))
    return hits / (len(gt) * k)


def coverage_at(pool_ids, gt, k):
    """Share of the true k nearest found anywhere in the pool: with best-k
    recall below it, the search reached the neighbours and the SQ8 distances
    ordered them below others; with both low, the graph did not reach them."""
    hits = 0
    for i in range(len(gt)):
        hits += len(set(pool_ids[i].tolist()) & set(gt[i, :k].tolist()))
    return hits / (len(gt) * k)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(self.device)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.6)  # let the sampler start before the timed region
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- helpers
def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            j = json.load(f)
        return float(j["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(kernel, name, ef):
    """The committed ncu capture of `kernel` on workload `name` at this ef
    (DRAM bytes per query, L2 sector hit rate), or None."""
    p = os.path.join(ROOT, "profiles", "search_traffic.json")
    try:
        with open(p) as f:
            rows = json.load(f)
    except Exception:
        return None
    for r in rows:
        if r.get("kernel") == kernel and r.get("workload") == name and r.get("ef") == ef:
            return r
    return None


def cpu_reference_search(path, w, queries, k, ef, nthreads):
    """The reference's own search (oracle/_ref) or the C oracle port."""
    from oracle.oracle import Oracle, RefHarness, read_index, ref_available

    if ref_available():
        try:
            h = RefHarness()
            r = h.open(path, w["n"], w["dim"], w["deg"])
            return (lambda q: r.search(q, k, ef, nthreads=nthreads)), "reference", r
        except OSError:
            pass
    o = Oracle(read_index(path, w["n"], w["dim"], w["deg"]))
    return (lambda q: o.search(q, k, ef, nthreads=nthreads, pool=False).compat), "port", o


def time_cpu(fn, queries, budget_s, min_q=256):
    """Times fn over a bounded sample sized for about budget_s seconds."""
    s = min(min_q, len(queries))
    t = time.perf_counter()
    fn(queries[:s])
    dt = time.perf_counter() - t
    m = int(min(len(queries), max(s, s * budget_s / max(dt, 1e-6))))
    t = time.perf_counter()
    out = fn(queries[:m])
    dt = time.perf_counter() - t
    return m / dt, m, dt, out


# ---------------------------------------------------------------- arms
def reference_arm(args, w, name):
    """The reference's own search on the host cores. This process loads no GPU
    code: the index file comes from the cache, from bench_data/ (assembled on
    the CPU) or, failing both, from a child process running the GPU builder."""
    base = gen_data(w, "base")
    queries = gen_data(w, "query")
    path = index_path(name, w)
    prep = "index file and ground truth from the cache (built earlier on this machine)"
    if not (os.path.exists(path) and os.path.exists(gt_path(name, w, 0, len(queries)))):
        prep = assemble_shipped(name, w, base) or prepare_in_child(name, w)
    gt = np.load(gt_path(name, w, 0, len(queries)))
    del base
    nthreads = os.cpu_count() or 1
    # same ef rule as the GPU arm, decided with the reference's own pools
    chosen, rec = w["efs"][-1], None
    sample = queries[:2000]
    for ef in w["efs"]:
        fn, kind, keep = cpu_reference_search(path, w, sample, ef, ef, nthreads)
        pool = fn(sample)  # k = ef: the whole pool, ascending
        rec = recall_at(pool, gt[:len(sample)], w["k"])
        if rec >= 0.95:
            chosen = ef
            break
    k = w["k"]
    fn, kind, keep = cpu_reference_search(path, w, queries, k, chosen, nthreads)
    for _ in range(args.warmup):
        fn(queries)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        fn(queries)
        times.append(time.perf_counter() - t)
    nq = len(queries)
    qps = nq * len(times) / sum(times)
    maps = []
    try:
        with open("/proc/self/maps") as f:
            maps = sorted({l.split()[-1] for l in f if l.rstrip().endswith(".so")
                           and l.split()[-1].startswith(ROOT)})
    except OSError:
        pass
    line = {
        "impl": "reference", "metric": METRIC, "value": qps, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_str(name, w, nq, k, chosen), "ef": chosen, "k": k,
                   "recall_at_10_pool": rec, "parallelism": f"{nthreads} host threads, "
                                                          "one reference search per query"},
        "cpu_baseline": {"value": qps, "unit": "queries/s", "cores": nthreads, "kind": kind,
                         "sample": f"all {nq} queries per step, k={k}, ef={chosen}"},
        "e2e": {"value": qps, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "index_prep": prep,
        "repo_libraries_mapped": [os.path.relpath(m, ROOT) for m in maps],
    }
    print(json.dumps(line), flush=True)


def gpu_arm(args, w, name, rank, world, device):
    import torch

    import liteqg_b200
    from liteqg_b200._capi import check, lib
    from liteqg_b200.replicas import max_over_ranks

    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    base = gen_data(w, "base")
    queries = gen_data(w, "query", rank)
    path, t_build = get_index_file(name, w, base, device)
    n, dim, deg, nq, k = w["n"], w["dim"], w["deg"], w["nq"], w["k"]
    if args.profile:
        # a profiling run holds only the index, the queries and the kernels'
        # work areas on the device: no ground truth, no ef selection, no
        # autotuning (ef from --ef, launch shape of --mode, default 6)
        del base
        ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
        ix.load(path)
        ef = args.ef or w["efs"][0]
        if args.profile_queries:
            # a smaller batch (e.g. one that runs one query per block)
            queries = queries[:args.profile_queries]
            nq = len(queries)
        c = FIXED_TUNING[args.mode or 6]
        ix.set_tuning(mode=c[0], lanes_per_cand=c[1], visited_bits=c[2], warps_per_block=c[3],
                      heap_warps=c[4], heap_scap=c[5])
        dev = torch.device("cuda", device)
        sh = torch.cuda.current_stream(dev).cuda_stream
        q_dev = torch.from_numpy(queries).to(dev)
        ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
        if args.fastscan:
            # the FastScan/RaBitQ search instead (its section encoded first)
            ix.fastscan_build(seed=0)
            search = lambda: ix.search_fastscan_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k,
                                                       ef=ef, stream=sh)
        else:
            search = lambda: ix.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k, ef=ef,
                                              stream=sh)
        search()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_push("lqg_profile")
        for _ in range(args.profile):
            search()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_pop()
        if args.fastscan:
            ix.fastscan_status(sh)
        else:
            ix.stream_status(sh)
        log(f"[rank {rank}] profiled {args.profile} steps, mode {c[0]}, ef {ef}, "
            f"fastscan {bool(args.fastscan)}")
        ix.close()
        return
    gt = ground_truth(name, w, base, queries, device, rank)
    log(f"[rank {rank}] data+index+gt ready in {time.perf_counter() - t0:.1f}s (build {t_build:.1f}s)")
    ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
    ix.load(path)
    log(f"[rank {rank}] index loaded {time.perf_counter() - t0:.1f}s")

    # ef selection on best-k-of-pool recall (untimed)
    chosen, recall = None, {}
    for ef in w["efs"]:
        _, (pid, _) = ix.search(queries, k, ef=ef, return_pool=True)
        recall[ef] = recall_at(pid, gt, k)
        if recall[ef] >= 0.95 and chosen is None:
            chosen = ef
            break
    if chosen is None:
        chosen = w["efs"][-1]
    ix.set_ef(chosen)
    log(f"[rank {rank}] ef={chosen} recall={recall} {time.perf_counter() - t0:.1f}s")
    knn_recall = None
    ref_built = None
    if w.get("knn_compare") and rank == 0:
        # the same search on the exact deg-NN graph of the same data (same
        # entry point, codes and parameters): what the builder's candidate
        # cap and the reference's omitted refine round could at most give
        knn_recall = knn_graph_recall(ix, w, gen_data(w, "base"), queries, gt, device)
        log(f"[rank {rank}] exact-kNN-graph recall {knn_recall}")
        ref_built = reference_built_recall(w, gen_data(w, "base"), queries, gt, device)
        log(f"[rank {rank}] reference-built index recall {ref_built}")

    dev = torch.device("cuda", device)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    q_dev = torch.from_numpy(queries).to(dev)
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    # exact-kernel pass: the reference's pops/evaluations (algorithmic bytes) and
    # a full-size parity check of the fast kernel against it
    ids_x = torch.empty((nq, k), dtype=torch.int32, device=dev)
    st = torch.zeros((nq, 4), dtype=torch.int32, device=dev)
    st_fast = torch.zeros((nq, 4), dtype=torch.int32, device=dev)
    ix.search_device(q_dev.data_ptr(), nq, k, ids_x.data_ptr(), k, ef=chosen,
                     stats_ptr=st.data_ptr(), stream=sh, exact=True)
    # mode 1 (fast kernel, heap kernel for tied queries): its tie flags give the
    # share of queries that meet equal distances
    c1 = FIXED_TUNING[1]
    ix.set_tuning(mode=c1[0], lanes_per_cand=c1[1], visited_bits=c1[2], warps_per_block=c1[3],
                  heap_warps=c1[4], heap_scap=c1[5])
    ix.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k, ef=chosen,
                     stats_ptr=st_fast.data_ptr(), stream=sh)
    ix.stream_status(sh)
    mismatch = int((ids != ids_x).any(1).sum().item())
    stx = st.cpu().numpy().astype(np.int64)
    stf = st_fast.cpu().numpy().astype(np.int64)
    pops, evals = stx[:, 0], stx[:, 1]
    exact_share = float((stf[:, 2] >= 1).mean())
    # launch shape and policy (fast+heap or heap-only, buffer sizes): autotuned
    # on the whole batch; every setting gives the same ids
    from liteqg_b200 import autotune

    if args.mode:
        # one fixed kernel mode (to time or profile that kernel)
        c = FIXED_TUNING[args.mode]
        ix.set_tuning(mode=c[0], lanes_per_cand=c[1], visited_bits=c[2], warps_per_block=c[3],
                      heap_warps=c[4], heap_scap=c[5])
        mode, mode_ms = args.mode, {str(list(c)): None}
    else:
        tuned = autotune.tune(ix, queries, chosen, k, path=None, device=device)
        mode = tuned["mode"]
        mode_ms = {str(c): t for t, c in tuned["all"]}
    # algorithmic bytes (per launch): neighbour rows of popped nodes, codes of
    # evaluated nodes (+ the entry), the query; SQ8 params once per CTA
    bytes_launch = float((pops * 4 * deg + (evals + 1) * dim + 4 * dim).sum())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step(evs=None):
        if evs:
            ix.set_kernel_events(evs[0].cuda_event, evs[1].cuda_event)
        ix.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k, ef=chosen, stream=sh)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize(dev)
    K = args.steps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    for a, b in kev:  # materialise the handles
        a.record(stream)
        b.record(stream)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(device) as clk:
        for i in range(K):
            flush.fill_(i & 0xFF)
            ev[i][0].record(stream)
            step(kev[i])
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
    ix.set_kernel_events(0, 0)
    ix.stream_status(sh)
    tune = ix.get_tuning()
    log(f"[rank {rank}] timed loop done {time.perf_counter() - t0:.1f}s")
    step_ms = [a.elapsed_time(b) for a, b in ev]
    kern_ms = [a.elapsed_time(b) for a, b in kev]
    total_s = max_over_ranks(sum(step_ms) / 1e3, device=dev)
    value = world * nq * K / total_s
    kern_avg_s = statistics.mean(kern_ms) / 1e3
    achieved = bytes_launch / kern_avg_s / 1e9
    peak, peak_kind = load_peaks()

    # e2e through the host-buffer C ABI: pinned queries in, ids out
    q_pin = torch.from_numpy(queries).pin_memory()
    ids_pin = torch.empty((nq, k), dtype=torch.int32).pin_memory()
    h = ix.handle
    e2e_ms = []
    for i in range(max(3, args.warmup) + K):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        check(lib().lqg_search_batch(h, q_pin.data_ptr(), nq, None, k, None, chosen,
                                     ids_pin.data_ptr(), k, None, None, 0, None, sh))
        b.record(stream)
        b.synchronize()
        if i >= max(3, args.warmup):
            e2e_ms.append(a.elapsed_time(b))
    e2e_total = max_over_ranks(sum(e2e_ms) / 1e3, device=dev)
    e2e = world * nq * K / e2e_total
    e2e_ok = bool((ids_pin.numpy() == ids.cpu().numpy()).all())

    log(f"[rank {rank}] e2e done {time.perf_counter() - t0:.1f}s")
    extra = {}
    if rank == 0 and world == 1:
        # the configuration's grid: k in {10, 100} x ef in the workload's ef
        # set, each point timed (device-resident, L2 flushed), with its
        # best-10-of-pool recall, the algorithmic roofline fraction of the
        # search kernel and its ids against the reference on a sample
        extra["grid"] = grid_points(ix, w, name, path, queries, q_dev, gt, flush, stream, peak)
        # the upstream FastScan/RaBitQ search on the same graph, beside the SQ8 path
        extra["fastscan"] = fastscan_leg(ix, w, queries, q_dev, gt, flush, stream, peak)
        # the same search on a 4x larger batch (these queries and three more
        # query seeds of the workload), L2 flushed: the kernel's throughput
        # with less of the batch's ramp and tail per query
        q4 = torch.from_numpy(np.concatenate([queries] + [gen_data(w, "query", r)
                                                          for r in (1, 2, 3)])).to(dev)
        ids4 = torch.empty((len(q4), k), dtype=torch.int32, device=dev)
        for _ in range(2):
            ix.search_device(q4.data_ptr(), len(q4), k, ids4.data_ptr(), k, ef=chosen, stream=sh)
        t4 = _timed(lambda: ix.search_device(q4.data_ptr(), len(q4), k, ids4.data_ptr(), k,
                                             ef=chosen, stream=sh), 5, flush, stream)
        extra["large_batch"] = {"queries": len(q4), "ms": t4, "qps": len(q4) / (t4 / 1e3)}
        del q4, ids4
        # plain: one query per launch through Index.search (the reference call form)
        P = min(1000, nq)
        lat = []
        for i in range(P + 20):
            t = time.perf_counter()
            ix.search(queries[i % nq], k)
            if i >= 20:
                lat.append(time.perf_counter() - t)
        plain_qps = P / sum(lat)
        extra["plain_qps"] = plain_qps
        extra["plain_p50_ms"] = 1e3 * float(np.percentile(lat, 50))
        extra["plain_p99_ms"] = 1e3 * float(np.percentile(lat, 99))
        extra["batched_over_plain"] = value / plain_qps
        log(f"[rank {rank}] plain done {time.perf_counter() - t0:.1f}s")
        # CPU baseline: the reference's own search on the host cores, bounded sample
        nthreads = os.cpu_count() or 1
        fn, kind, keep = cpu_reference_search(path, w, queries, k, chosen, nthreads)
        cpu_qps, m, dt, cpu_ids = time_cpu(fn, queries, budget_s=8.0)
        ref_mismatch = int((cpu_ids[:m] != ids.cpu().numpy().view(np.uint32)[:m]).any(1).sum())
        # one host thread, one query per call (the reference's own timing
        # loop, reproduce/run.py:90-95)
        fn1, _, keep1 = cpu_reference_search(path, w, queries, k, chosen, 1)
        one = []
        for i in range(min(300, nq)):
            t = time.perf_counter()
            fn1(queries[i:i + 1])
            one.append(time.perf_counter() - t)
        cpu = {"value": cpu_qps, "unit": "queries/s", "cores": nthreads, "kind": kind,
               "sample": f"first {m} of {nq} queries, k={k}, ef={chosen}, {dt:.1f}s wall",
               "ids_mismatch_vs_gpu": ref_mismatch,
               "single_thread_per_call": {"queries": len(one),
                                          "p50_ms": 1e3 * float(np.median(one)),
                                          "qps": len(one) / sum(one)}}
    else:
        cpu = None

    kernel = {2: "heap_search_kernel", 4: "split_search_kernel", 5: "batch_search_kernel",
              6: "batch_search_kernel (lazy search heap)"}.get(mode)
    cap = profile_traffic(kernel, name, chosen) if kernel else None
    traffic_launch = cap["dram_bytes_per_query"] * nq if cap else None
    l2_hit = cap.get("l2_hit_rate") if cap else None
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": K,
        "warmup": max(3, args.warmup), "ms_per_step": statistics.mean(step_ms),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload_str(name, w, nq, k, chosen), "ef": chosen, "k": k,
                   "recall_at_10_pool": recall.get(chosen), "recall_by_ef": recall,
                   **({"recall_by_ef_exact_knn_graph": knn_recall} if knn_recall else {}),
                   **({"reference_built_index": ref_built} if ref_built else {}),
                   "l2": "flushed between steps (256 MiB write)", "parallelism": f"replicas x{world}",
                   "tuning": tune, "autotune_ms": mode_ms, "tied_query_share": exact_share,
                   "fast_vs_exact_id_mismatch": mismatch, "e2e_ids_equal": e2e_ok,
                   "pops_mean": float(pops.mean()), "evals_mean": float(evals.mean())},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic_launch, "l2_hit_rate": l2_hit,
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "kernel_ms": statistics.mean(kern_ms),
                     "kernel": {1: "fast_search_kernel + heap_search_kernel (tied queries)",
                                2: "heap_search_kernel",
                                4: "split_search_kernel",
                                5: "batch_search_kernel",
                                6: "batch_search_kernel (lazy search heap)"}.get(mode, str(mode))},
        "e2e": {"value": e2e, "unit": "queries/s", "h2d_bytes_per_step": int(nq * dim * 4),
                "d2h_bytes_per_step": int(nq * k * 4)},
        # kernels per batched step: fast + heap + exact (1), heap + exact (2),
        # per step: the work order (entry-distance kernel + 4 radix-sort
        # passes compiled into the library from CUB), then fast + heap + exact
        # (1), heap + exact (2), replay + result replay + exact (3), split or
        # batch + exact (4-6); the L2 flush is torch's
        "gpu_launches": (5 + {1: 3, 2: 2, 3: 3, 4: 2, 5: 2, 6: 2}.get(mode, 3)) * K,
        "clocks": clk.summary(),
        "p50_ms": statistics.median(step_ms), "p99_ms": float(np.percentile(step_ms, 99)),
        **extra,
    }
    if cpu is not None:
        line["cpu_baseline"] = cpu
    if rank == 0:
        print(json.dumps(line), flush=True)
    ix.close()


def knn_graph_recall(ix, w, base, queries, gt, device):
    """Best-10-of-pool recall by ef of the same search on the exact deg-NN
    graph of the base vectors (FP32 on the GPU), entry point, codes and SQ8
    parameters of `ix`."""
    import torch

    import liteqg_b200

    dev = torch.device("cuda", device)
    xb = torch.from_numpy(base).to(dev)
    nb2 = (xb * xb).sum(1)
    deg = w["deg"]
    nbrs = np.empty((len(base), deg), np.uint32)
    for s0 in range(0, len(base), 4096):
        q = xb[s0:s0 + 4096]
        d = nb2[None, :] - 2.0 * (q @ xb.T) + (q * q).sum(1)[:, None]
        d[torch.arange(len(q), device=dev), torch.arange(s0, s0 + len(q), device=dev)] = float("inf")
        nbrs[s0:s0 + len(q)] = torch.topk(d, deg, dim=1, largest=False).indices.cpu().numpy()
    del xb
    entry, vecs, _, codes, params = ix.get_arrays()
    kx = liteqg_b200.Index("QG", "L2", w["n"], w["dim"], deg, device=device)
    kx.set_arrays(entry, vecs, nbrs, codes, params)
    out = {}
    for ef in w["efs"]:
        _, (pid, _) = kx.search(queries, 10, ef=ef, return_pool=True)
        out[ef] = recall_at(pid, gt, 10)
    kx.close()
    return out


def reference_built_recall(w, base, queries, gt, device):
    """Best-10-of-pool recall by ef of the same search (this package's, exact
    against the reference) on an index built from the same base vectors by
    the reference's own builder (QGBuilder, compiled from its sources into
    oracle/_ref, on all host cores), and the build's wall time; None when
    oracle/_ref is absent."""
    import tempfile

    import liteqg_b200
    from oracle.oracle import RefHarness, ref_available

    if not ref_available():
        return None
    path = os.path.join(tempfile.mkdtemp(), "reference_built.idx")
    # the reference's builder prints its progress on stdout, which carries
    # only this program's JSON line: point file descriptor 1 at stderr
    sys.stdout.flush()
    saved = os.dup(1)
    os.dup2(2, 1)
    try:
        t = time.perf_counter()
        RefHarness().build(base, w["deg"], w["efb"], w["iters"], path,
                           nthreads=os.cpu_count() or 1)
        build_s = time.perf_counter() - t
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
    rx = liteqg_b200.Index("QG", "L2", w["n"], w["dim"], w["deg"], device=device)
    rx.load(path)
    out = {}
    for ef in w["efs"]:
        _, (pid, _) = rx.search(queries, 10, ef=ef, return_pool=True)
        out[ef] = recall_at(pid, gt, 10)
    rx.close()
    os.remove(path)
    return {"recall_by_ef": out, "build_s": build_s, "threads": os.cpu_count() or 1}


def grid_points(ix, w, name, path, queries, q_dev, gt, flush, stream, peak):
    """k x ef grid of the headline workload (see gpu_arm)."""
    import torch

    nq, dim, deg = len(queries), w["dim"], w["deg"]
    sh = stream.cuda_stream
    dev = q_dev.device
    nthreads = os.cpu_count() or 1
    sample = min(1000, nq)
    out = {}
    for ef in w["efs"]:
        st = torch.zeros((nq, 4), dtype=torch.int32, device=dev)
        idx = torch.empty((nq, 1), dtype=torch.int32, device=dev)
        ix.search_device(q_dev.data_ptr(), nq, 1, idx.data_ptr(), 1, ef=ef,
                         stats_ptr=st.data_ptr(), stream=sh, exact=True)
        stx = st.cpu().numpy().astype(np.int64)
        bytes_launch = float((stx[:, 0] * 4 * deg + (stx[:, 1] + 1) * dim + 4 * dim).sum())
        _, (pid, _) = ix.search(queries, 10, ef=ef, return_pool=True)
        rec = recall_at(pid, gt, 10)
        for k in (10, w["k_extra"]):
            ids = torch.empty((nq, k), dtype=torch.int32, device=dev)

            def run():
                ix.search_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k, ef=ef, stream=sh)

            for _ in range(2):
                run()
            ix.stream_status(sh)
            reps, step_ms, kern_ms = 5, [], []
            for i in range(reps):
                flush.fill_(i & 0xFF)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ka, kb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ka.record(stream)  # materialise the handles the library records into
                kb.record(stream)
                ix.set_kernel_events(ka.cuda_event, kb.cuda_event)
                a.record(stream)
                run()
                b.record(stream)
                b.synchronize()
                step_ms.append(a.elapsed_time(b))
                kern_ms.append(ka.elapsed_time(kb))
            ix.set_kernel_events(0, 0)
            ix.stream_status(sh)
            fn, kind, keep = cpu_reference_search(path, w, queries[:sample], k, ef, nthreads)
            ref_ids = fn(queries[:sample])
            got = ids.cpu().numpy().view(np.uint32)[:sample]
            achieved = bytes_launch / (statistics.mean(kern_ms) / 1e3) / 1e9
            out[f"k{k}_ef{ef}"] = {
                "qps": nq / (statistics.mean(step_ms) / 1e3), "ms": statistics.mean(step_ms),
                "recall_at_10_pool": rec, "roofline_frac": achieved / peak,
                "achieved_gbs": achieved, "pops_mean": float(stx[:, 0].mean()),
                "evals_mean": float(stx[:, 1].mean()),
                "ids_mismatch_vs_reference": int((ref_ids != got).any(1).sum()),
                "reference_sample": f"first {sample} queries ({kind})"}
            log(f"[grid] k={k} ef={ef}: {out[f'k{k}_ef{ef}']}")
    return out


def fastscan_leg(ix, w, queries, q_dev, gt, flush, stream, peak):
    """The upstream FastScan/RaBitQ search (search_qg with an exact re-rank of
    every popped node) on the headline index: its section encoded on the GPU
    (lqg_fs_build), then for each ef: device-resident QPS (L2 flushed),
    recall@10 of its k = 10 output, the roofline fraction of its algorithmic
    bytes (one row per expanded node, a vector and ids row per update_results
    evaluation, the query), ids against the reference's own search_qg on a
    sample, and that reference's CPU throughput on all host cores."""
    import torch

    from oracle.oracle import RefFastScan, ref_available

    nq, dim, deg = len(queries), w["dim"], w["deg"]
    sh = stream.cuda_stream
    dev = q_dev.device
    torch.cuda.synchronize(dev)
    t = time.perf_counter()
    ix.fastscan_build(seed=0)
    enc_s = time.perf_counter() - t
    diag, packed, fac = ix.fastscan_arrays()
    P = len(diag)
    row_bytes = 4 * ((dim + 3) & ~3) + deg * P // 8 + 16 * deg
    ref = None
    if ref_available():
        _, vecs, nbrs, _, _ = ix.get_arrays()
        ref = RefFastScan().open(w["n"], dim, deg, ix.entry_point(), vecs, nbrs, packed, fac, diag)
        del vecs
    del packed, fac
    k = 10
    out = {"encode_s": enc_s, "row_bytes": row_bytes, "padded_dim": P, "points": {}}
    ids = torch.empty((nq, k), dtype=torch.int32, device=dev)
    st = torch.zeros((nq, 4), dtype=torch.int32, device=dev)
    nthreads = os.cpu_count() or 1
    for ef in (16, 32, 64, 128):
        def run():
            ix.search_fastscan_device(q_dev.data_ptr(), nq, k, ids.data_ptr(), k, ef=ef,
                                      stats_ptr=st.data_ptr(), stream=sh)

        for _ in range(2):
            run()
        ix.fastscan_status(sh)
        ms = _timed(run, 5, flush, stream)
        ix.fastscan_status(sh)
        got = ids.cpu().numpy().view(np.uint32)
        stx = st.cpu().numpy().astype(np.int64)
        bytes_launch = float((stx[:, 1] * row_bytes + stx[:, 2] * (4 * dim + 4 * deg) + 4 * dim).sum())
        pt = {"qps": nq / (ms / 1e3), "ms": ms, "recall_at_10": recall_at(got, gt, 10),
              "roofline_frac": bytes_launch / (ms / 1e3) / 1e9 / peak,
              "algorithmic_bytes_per_launch": bytes_launch,
              "expanded_mean": float(stx[:, 1].mean()), "pops_mean": float(stx[:, 0].mean()),
              "pops_p99": float(np.percentile(stx[:, 0], 99)), "pops_max": int(stx[:, 0].max())}
        if ref is not None:
            sample = min(1000, nq)
            r_ids = ref.search(queries[:sample], k, ef, nthreads)
            pt["ids_mismatch_vs_reference"] = int((r_ids != got[:sample]).any(1).sum())
            qps, m, dt, _ = time_cpu(lambda qq: ref.search(qq, k, ef, nthreads), queries, 3.0)
            pt["cpu_reference_qps"] = qps
            pt["cpu_reference_sample"] = f"first {m} queries, {nthreads} threads, {dt:.1f}s"
        out["points"][str(ef)] = pt
        log(f"[fastscan] ef={ef}: {pt}")
    if ref is not None:
        ref.close()
    return out


def _timed(fn, reps, flush, stream):
    """Mean device ms of fn over reps, L2 flushed before each (CUDA events)."""
    import torch

    tot = 0.0
    for i in range(reps):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        b.synchronize()
        tot += a.elapsed_time(b)
    return tot / reps


def uneven_arm(args, w, name, device):
    """The uneven high-dimension batch: one batch with per-query ef and k, eager
    and as a CUDA graph."""
    import torch

    import liteqg_b200

    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    base = gen_data(w, "base")
    queries = gen_data(w, "query")
    path, t_build = get_index_file(name, w, base, device)
    n, dim, deg, nq = w["n"], w["dim"], w["deg"], w["nq"]
    rng = np.random.default_rng(2)
    efq = rng.choice(w["ef_choices"], nq).astype(np.uint32)
    kq = rng.choice(w["k_choices"], nq).astype(np.uint32)
    kmax, efmax = int(kq.max()), int(efq.max())
    if args.profile:
        # profiling: only the index, the queries and the kernels' work areas
        # on the device; the launch shape of --mode (default 2, the heap kernel)
        del base
        ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
        ix.load(path)
        mode = args.mode or 2
        ix.set_tuning(mode=mode, lanes_per_cand=2, heap_warps=4, heap_scap=512, visited_bits=10)
        dev = torch.device("cuda", device)
        sh = torch.cuda.current_stream(dev).cuda_stream
        q_dev = torch.from_numpy(queries).to(dev)
        ids = torch.empty((nq, kmax), dtype=torch.int32, device=dev)
        e_dev = torch.from_numpy(efq.view(np.int32)).to(dev)
        k_dev = torch.from_numpy(kq.view(np.int32)).to(dev)
        run = lambda: ix.search_device(q_dev.data_ptr(), nq, 0, ids.data_ptr(), kmax, ef=efmax,
                                       ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(), stream=sh)
        run()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_push("lqg_profile")
        for _ in range(args.profile):
            run()
        torch.cuda.synchronize(dev)
        torch.cuda.nvtx.range_pop()
        ix.stream_status(sh)
        log(f"[uneven] profiled {args.profile} steps, mode {mode}")
        return
    gt = ground_truth(name, w, base, queries, device, 0)
    del base
    log(f"[uneven] index + gt ready {time.perf_counter() - t0:.1f}s (build {t_build:.1f}s)")
    ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
    ix.load(path)
    # recall: best-10 of each query's pool (untimed)
    _, (pid, _) = ix.search(queries, 10, ef=efq, return_pool=True)
    rec_by_ef = {int(e): recall_at(pid[efq == e], gt[efq == e], 10) for e in w["ef_choices"]}
    cov_by_ef = {int(e): coverage_at(pid[efq == e], gt[efq == e], 10) for e in w["ef_choices"]}
    dev = torch.device("cuda", device)
    stream = torch.cuda.current_stream(dev)
    sh = stream.cuda_stream
    q_dev = torch.from_numpy(queries).to(dev)
    ids = torch.empty((nq, kmax), dtype=torch.int32, device=dev)
    e_dev = torch.from_numpy(efq.view(np.int32)).to(dev)
    k_dev = torch.from_numpy(kq.view(np.int32)).to(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def step():
        ix.search_device(q_dev.data_ptr(), nq, 0, ids.data_ptr(), kmax, ef=efmax,
                         ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(), stream=sh)

    best = None
    # (mode, lanes per candidate, heap warps per block, heap slots, visited
    # bits[, 1: batch kernels one query per block of 4 warps])
    shapes = ((6, 2, 4, 512, 10), (6, 4, 4, 512, 10), (5, 2, 4, 512, 10), (4, 4, 4, 512, 10),
              (2, 2, 4, 512, 10), (2, 4, 4, 512, 10), (1, 4, 4, 512, 10),
              (2, 2, 4, 256, 10), (2, 2, 4, 256, 9), (2, 2, 2, 512, 10), (2, 2, 8, 256, 9),
              # larger visited caches: fewer forgotten nodes evaluated again at
              # ef up to 512, against fewer resident warps
              (2, 2, 2, 512, 12), (2, 2, 4, 256, 11), (2, 2, 2, 256, 13), (2, 2, 3, 512, 12),
              # the query-per-block form on the whole batch: 960-byte rows make
              # the distances most of a pop, which its 4 warps share
              (6, 4, 4, 512, 10, 1), (6, 4, 4, 512, 11, 1), (6, 4, 4, 512, 12, 1),
              (5, 4, 4, 512, 11, 1))
    from liteqg_b200._capi import SMALL_BATCH_AUTO, LqgError

    for shape in shapes:
        mode, g, hw, scap, vb = shape[:5]
        cta = len(shape) > 5 and shape[5]
        ix.set_tuning(mode=mode, lanes_per_cand=g, heap_warps=hw, heap_scap=scap, visited_bits=vb,
                      small_batch=nq if cta else SMALL_BATCH_AUTO)
        try:
            for _ in range(2):
                step()
            ix.stream_status(sh)
        except LqgError as e:  # a launch shape this index's size cannot take
            log(f"[uneven] shape {shape} skipped: {e}")
            continue
        ms = _timed(step, 5, flush, stream)
        log(f"[uneven] mode {mode} G {g} warps {hw} scap {scap} vbits {vb} "
            f"{'block per query ' if cta else ''}: {ms:.2f} ms")
        if best is None or ms < best[0]:
            best = (ms, shape)
    mode, g, hw, scap, vb = best[1][:5]
    cta = len(best[1]) > 5 and best[1][5]
    best = (best[0], mode, g, hw, scap, vb, bool(cta))
    ix.set_tuning(mode=mode, lanes_per_cand=g, heap_warps=hw, heap_scap=scap, visited_bits=vb,
                  small_batch=nq if cta else SMALL_BATCH_AUTO)
    for _ in range(max(3, args.warmup)):
        step()
    ix.stream_status(sh)
    K = max(1, min(args.steps, 50))
    eager_ms, kern_ms = [], []
    for i in range(K):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ka, kb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ka.record(stream)  # materialise the handles the library records into
        kb.record(stream)
        ix.set_kernel_events(ka.cuda_event, kb.cuda_event)
        a.record(stream)
        step()
        b.record(stream)
        b.synchronize()
        eager_ms.append(a.elapsed_time(b))
        kern_ms.append(ka.elapsed_time(kb))
    ix.set_kernel_events(0, 0)
    ix.stream_status(sh)
    eager_ms = statistics.mean(eager_ms)
    eager_ids = ids.cpu().numpy().copy()
    # the reference's work per query (pops, evaluations; the exact kernel
    # counts them exactly) for the algorithmic bytes of the launch
    stx = torch.zeros((nq, 4), dtype=torch.int32, device=dev)
    idx = torch.empty((nq, kmax), dtype=torch.int32, device=dev)
    ix.search_device(q_dev.data_ptr(), nq, 0, idx.data_ptr(), kmax, ef=efmax,
                     ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(), stats_ptr=stx.data_ptr(),
                     stream=sh, exact=True)
    ix.stream_status(sh)
    stx = stx.cpu().numpy().astype(np.int64)
    pops, evals = stx[:, 0], stx[:, 1]
    bytes_launch = float((pops * 4 * deg + (evals + 1) * dim + 4 * dim).sum())
    achieved = bytes_launch / (statistics.mean(kern_ms) / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    # e2e through the host-buffer C ABI with the per-query k and ef arrays
    from liteqg_b200._capi import check, lib

    q_pin = torch.from_numpy(queries).pin_memory()
    ids_pin = torch.empty((nq, kmax), dtype=torch.int32).pin_memory()
    k_pin = torch.from_numpy(kq.view(np.int32)).pin_memory()
    e_pin = torch.from_numpy(efq.view(np.int32)).pin_memory()
    e2e_ms = []
    for i in range(2 + K):
        flush.fill_(i & 0xFF)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        check(lib().lqg_search_batch(ix.handle, q_pin.data_ptr(), nq, k_pin.data_ptr(), 0,
                                     e_pin.data_ptr(), efmax, ids_pin.data_ptr(), kmax, None,
                                     None, 0, None, sh))
        b.record(stream)
        b.synchronize()
        if i >= 2:
            e2e_ms.append(a.elapsed_time(b))
    e2e_qps = nq / (statistics.mean(e2e_ms) / 1e3)
    col = np.arange(kmax)[None, :] < kq[:, None]
    e2e_ok = bool((ids_pin.numpy()[col] == eager_ids[col]).all())
    # CPU baseline: the compiled reference on all host cores, the whole batch
    # (grouped by (ef, k), its search takes one of each per call)
    nthreads = os.cpu_count() or 1
    ref_ids = np.full((nq, kmax), 0xFFFFFFFF, np.uint32)
    t_cpu, kind = 0.0, None
    for e in w["ef_choices"]:
        for kk in w["k_choices"]:
            sel = np.nonzero((efq == e) & (kq == kk))[0]
            if len(sel) == 0:
                continue
            fn, kind, keep = cpu_reference_search(path, w, queries[sel], int(kk), int(e), nthreads)
            t = time.perf_counter()
            out = fn(queries[sel])
            t_cpu += time.perf_counter() - t
            ref_ids[sel, :kk] = out
    got = eager_ids.view(np.uint32)
    ref_mismatch = int(((ref_ids != got) & col).any(1).sum())
    cpu = {"value": nq / t_cpu, "unit": "queries/s", "cores": nthreads, "kind": kind,
           "sample": f"all {nq} queries, each at its own ef and k, {t_cpu:.1f}s wall",
           "ids_mismatch_vs_gpu": ref_mismatch}
    log(f"[uneven] cpu {cpu}")
    # the same batch captured in a CUDA graph
    s2 = torch.cuda.Stream(dev)
    s2.wait_stream(stream)
    with torch.cuda.stream(s2):
        ix.search_device(q_dev.data_ptr(), nq, 0, ids.data_ptr(), kmax, ef=efmax,
                         ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(), stream=s2.cuda_stream)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph, stream=s2):
            ix.search_device(q_dev.data_ptr(), nq, 0, ids.data_ptr(), kmax, ef=efmax,
                             ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(),
                             stream=s2.cuda_stream)
    torch.cuda.synchronize(dev)
    graph_ms = _timed(graph.replay, K, flush, stream)
    graph_ok = bool((ids.cpu().numpy() == eager_ids).all())
    del graph
    line = {
        "metric": METRIC, "value": nq / (eager_ms / 1e3), "unit": "queries/s", "n_gpus": 1,
        "steps": K, "warmup": max(3, args.warmup), "ms_per_step": eager_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{name}: N={n} D={dim} deg={deg} EF={w['efb']}, {nq} queries, "
                               f"per-query ef from {list(w['ef_choices'])}, k from "
                               f"{list(w['k_choices'])} (seed 2)",
                   "recall_at_10_pool_by_ef": rec_by_ef, "pool_coverage_at_10_by_ef": cov_by_ef,
                   "mode": best[1], "lanes_per_cand": 4 if best[6] else best[2],
                   "warps_per_block": 4 if best[6] else best[3], "heap_scap": best[4],
                   "visited_bits": best[5], "query_per_block": best[6],
                   "l2": "flushed between steps (256 MiB write)"},
        "graph_qps": nq / (graph_ms / 1e3), "graph_ids_equal": graph_ok,
        "gpu_launches": (5 + {1: 3, 2: 2, 3: 3, 4: 2, 5: 2, 6: 2}.get(best[1], 3)) * K,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "kernel_ms": statistics.mean(kern_ms),
                     "kernel": {1: "fast_search_kernel + heap_search_kernel (tied queries)",
                                2: "heap_search_kernel", 4: "split_search_kernel",
                                5: "batch_search_kernel",
                                6: "batch_search_kernel (lazy search heap)"}.get(best[1]) +
                               (", one query per block of 4 warps" if best[6] else "")},
        "e2e": {"value": e2e_qps, "unit": "queries/s",
                "h2d_bytes_per_step": int(nq * dim * 4 + 8 * nq),
                "d2h_bytes_per_step": int(nq * kmax * 4), "ids_equal": e2e_ok},
        "cpu_baseline": cpu,
        "pops_mean": float(pops.mean()), "evals_mean": float(evals.mean()),
    }
    print(json.dumps(line), flush=True)


SERVING_STREAMS = 8  # batches in flight at once (each on its own stream)


def serving_arm(args, w, name, device):
    """The serving workload: open-loop Poisson arrivals through the serving loop."""
    import torch

    import liteqg_b200
    from liteqg_b200.serving import Server

    torch.cuda.set_device(device)
    t0 = time.perf_counter()
    base = gen_data(w, "base")
    queries = gen_data(w, "query")
    path, t_build = get_index_file(name, w, base, device)
    sample = queries[:2000]
    gt = ground_truth(name, w, base, sample, device, 0)
    del base
    log(f"[serving] index + gt ready {time.perf_counter() - t0:.1f}s (build {t_build:.1f}s)")
    n, dim, deg = w["n"], w["dim"], w["deg"]
    ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
    ix.load(path)
    # kernel mode: the fastest on one 8,192-query batch of the request mix
    # (every mode returns the same ids)
    rng = np.random.default_rng(4)
    mq = 8192
    q_dev = torch.from_numpy(queries[:mq]).cuda(device)
    k_dev = torch.from_numpy(rng.choice(w["k_choices"], mq).astype(np.uint32)).cuda(device)
    e_dev = torch.from_numpy(rng.choice(w["ef_choices"], mq).astype(np.uint32)).cuda(device)
    kmax, efmax = max(w["k_choices"]), max(w["ef_choices"])
    ids = torch.empty((mq, kmax), dtype=torch.int32, device=q_dev.device)
    stream = torch.cuda.current_stream(q_dev.device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=q_dev.device)

    def step():
        ix.search_device(q_dev.data_ptr(), mq, 0, ids.data_ptr(), kmax, ef=efmax,
                         ef_ptr=e_dev.data_ptr(), k_ptr=k_dev.data_ptr(),
                         stream=stream.cuda_stream)

    best = None
    for mode, g in ((6, 2), (5, 2), (4, 4), (2, 2), (2, 4)):
        ix.set_tuning(mode=mode, lanes_per_cand=g, heap_warps=4, heap_scap=512, visited_bits=10)
        step()
        ix.stream_status(stream.cuda_stream)
        ms = _timed(step, 3, flush, stream)
        log(f"[serving] mode {mode} G {g}: {ms:.2f} ms per {mq} mixed requests")
        if best is None or ms < best[0]:
            best = (ms, mode, g)
    ix.set_tuning(mode=best[1], lanes_per_cand=best[2], heap_warps=4, heap_scap=512,
                  visited_bits=10)
    del q_dev, k_dev, e_dev, ids, flush
    rec, cov = {}, {}
    for ef in w["ef_choices"]:
        _, (pid, _) = ix.search(sample, 10, ef=ef, return_pool=True)
        rec[int(ef)] = recall_at(pid, gt, 10)
        cov[int(ef)] = coverage_at(pid, gt, 10)
    rng = np.random.default_rng(3)
    rows = []
    with Server(ix, streams=SERVING_STREAMS, max_k=max(w["k_choices"]),
                max_ef=max(w["ef_choices"])) as srv:
        for rate in w["rates"]:
            m = int(min(len(queries), rate * w["seconds"]))
            arrivals = np.cumsum(rng.exponential(1e6 / rate, m))
            ks = rng.choice(w["k_choices"], m).astype(np.uint32)
            efs = rng.choice(w["ef_choices"], m).astype(np.uint32)
            srv.reset_stats()
            t = time.perf_counter()
            sids, lat = srv.replay(queries[:m], ks, efs, arrivals)
            wall = time.perf_counter() - t
            st = srv.stats()
            # ids of a sample of the served requests against the reference's
            # own search of each alone (its k and ef)
            samp = rng.choice(m, min(m, 1000), replace=False)
            mism = 0
            for e in w["ef_choices"]:
                for kk in w["k_choices"]:
                    sel = samp[(efs[samp] == e) & (ks[samp] == kk)]
                    if len(sel) == 0:
                        continue
                    fn, kind, keep = cpu_reference_search(path, w, queries[sel], int(kk), int(e),
                                                          os.cpu_count() or 1)
                    mism += int((fn(queries[sel]) != sids[sel, :kk]).any(1).sum())
            # served rate: requests over the time from the first scheduled
            # arrival to the last completion (arrival + latency, both measured
            # by the server from the call's start); the wall time around the
            # call also holds the Python-side set-up of the request arrays
            span_s = float(np.max(arrivals + lat)) / 1e6
            rows.append({"offered_qps": rate, "requests": m, "achieved_qps": m / span_s,
                         "call_wall_s": wall,
                         "p50_ms": float(np.percentile(lat, 50)) / 1e3,
                         "p99_ms": float(np.percentile(lat, 99)) / 1e3,
                         "mean_batch": st["mean_batch"],
                         "ids_mismatch_vs_reference": mism,
                         "reference_sample": f"{len(samp)} served requests ({kind})"})
            log(f"[serving] {rows[-1]}")
    # plain path: one query per call
    lat = []
    for i in range(520):
        t = time.perf_counter()
        ix.search(queries[i], 10, ef=100)
        if i >= 20:
            lat.append(time.perf_counter() - t)
    line = {
        "metric": METRIC, "value": max(r["achieved_qps"] for r in rows), "unit": "queries/s",
        "n_gpus": 1, "steps": len(rows), "warmup": 0, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": f"{name}: N={n} D={dim} deg={deg} EF={w['efb']}, open-loop "
                               f"Poisson arrivals, k from {list(w['k_choices'])}, ef from "
                               f"{list(w['ef_choices'])}", "recall_at_10_pool_by_ef": rec,
                   "pool_coverage_at_10_by_ef": cov,
                   "server": {"streams": SERVING_STREAMS, "mode": best[1],
                              "lanes_per_cand": best[2]}},
        "serving": rows,
        "plain_qps": len(lat) / sum(lat), "plain_p50_ms": 1e3 * float(np.percentile(lat, 50)),
        "plain_p99_ms": 1e3 * float(np.percentile(lat, 99)),
    }
    print(json.dumps(line), flush=True)


def build_arm(args, w, name, device):
    """The build workload: the same data built twice, with the BF16 tensor-core
    prune (pair_kernel 1) and with the FP32 prune (pair_kernel 0); reports the
    build times, the share of pruned edges that differ, recall@10 (best 10 of
    the pool) of the queries at the workload's ef on both indexes, and the
    error of the two distance forms against FP64 on sampled candidate sets."""
    import torch

    import liteqg_b200

    torch.cuda.set_device(device)
    base = gen_data(w, "base")
    queries = gen_data(w, "query")
    n, dim, deg, ef = w["n"], w["dim"], w["deg"], w["ef"]
    res, graphs = {}, {}
    for label, pk in (("bf16_tensor_core", 1), ("fp32", 0)):
        ix = liteqg_b200.Index("QG", "L2", n, dim, deg, device=device)
        t = time.perf_counter()
        rep = ix.build_index(base, w["efb"], num_iter=w["iters"], random_edges=w["random_edges"],
                             path_take=w["path_take"], far_budget=w["far_budget"], pair_kernel=pk)
        wall = time.perf_counter() - t
        _, (pid, _) = ix.search(queries, 10, ef=ef, return_pool=True)
        graphs[label] = ix.get_arrays()[2]
        res[label] = {"build_s": wall, "report": rep, "pool": pid}
        ix.close()
        log(f"[build] {label}: {wall:.1f}s {rep}")
    gt = ground_truth(name, w, base, queries, device, 0)
    for label in res:
        res[label]["recall_at_10"] = recall_at(res[label].pop("pool"), gt, 10)

    def edges(nb):
        src = np.repeat(np.arange(n, dtype=np.int64), deg)
        dst = nb.reshape(-1).astype(np.int64)
        ok = dst < n
        return np.unique(src[ok] * n + dst[ok])

    ea, eb = edges(graphs["bf16_tensor_core"]), edges(graphs["fp32"])
    common = np.intersect1d(ea, eb, assume_unique=True).size
    disagree = 1.0 - common / max(1, ea.size)

    # distance error against FP64 on the neighbour sets of sampled nodes (the
    # sets the prune compares), emulated with torch: BF16-rounded rows centred
    # on the set's mean, exact products summed in FP32, FP32 norms (the tensor
    # core form), and the FP32 sum of squared differences (the FP32 prune)
    rng = np.random.default_rng(5)
    dev = torch.device("cuda", device)
    nb = graphs["bf16_tensor_core"]
    rel_tc, rel_32 = [], []
    for u in rng.choice(n, 500, replace=False):
        ids = nb[u][nb[u] < n]
        x = torch.from_numpy(base[ids]).to(dev)
        x64 = x.double()
        d64 = torch.cdist(x64, x64) ** 2
        c = x - x.mean(0, keepdim=True)
        cb = c.bfloat16().float()
        nrm = (c * c).sum(1)
        dtc = nrm[:, None] + nrm[None, :] - 2.0 * (cb @ cb.T)
        d32 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(2)
        iu = torch.triu_indices(len(ids), len(ids), 1, device=dev)
        ref = d64[iu[0], iu[1]]
        rel_tc.append(((dtc.double()[iu[0], iu[1]] - ref).abs() / ref).cpu().numpy())
        rel_32.append(((d32.double()[iu[0], iu[1]] - ref).abs() / ref).cpu().numpy())
    rel_tc, rel_32 = np.concatenate(rel_tc), np.concatenate(rel_32)

    tc = res["bf16_tensor_core"]
    line = {
        "metric": "index build: nodes/s with the BF16 tensor-core prune", "value": n / tc["build_s"],
        "unit": "nodes/s", "n_gpus": 1, "steps": 1, "warmup": 0, "ms_per_step": 1e3 * tc["build_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "bf16 (prune Gram), f32",
        "data": "synthetic",
        "config": {"workload": f"{name}: N={n} D={dim} unit-length rows from a Gaussian mixture of "
                               f"{w['clusters']} clusters (sigma {w['sigma']}), deg={deg}, EF={w['efb']}, "
                               f"{w['iters']} rounds; {w['nq']} queries, recall@10 at ef={ef}"},
        "builds": res,
        "pruned_edge_disagreement": disagree, "edges": int(ea.size),
        "distance_rel_error_vs_fp64": {
            "pairs": int(rel_tc.size), "sample": "all pairs of the final neighbour lists of 500 nodes "
                                                 "(emulated on the GPU with torch)",
            "bf16_gram": {"median": float(np.median(rel_tc)), "p99": float(np.percentile(rel_tc, 99)),
                          "max": float(rel_tc.max())},
            "fp32": {"median": float(np.median(rel_32)), "p99": float(np.percentile(rel_32, 99)),
                     "max": float(rel_32.max())}},
    }
    print(json.dumps(line), flush=True)


def build_only(w, name, device):
    """One GPU build of the workload's index inside an NVTX range 'lqg_build'
    (the range a profiler filters on); prints the build report as JSON."""
    import torch

    import liteqg_b200

    base = gen_data(w, "base")
    ix = liteqg_b200.Index("QG", "L2", w["n"], w["dim"], w["deg"], device=device)
    torch.cuda.nvtx.range_push("lqg_build")
    t = time.perf_counter()
    rep = ix.build_index(base, w["efb"], num_iter=w["iters"], random_edges=w["random_edges"],
                         path_take=w["path_take"], far_budget=w["far_budget"])
    wall = time.perf_counter() - t
    torch.cuda.nvtx.range_pop()
    ix.close()
    print(json.dumps({"workload": name, "n": w["n"], "dim": w["dim"], "deg": w["deg"],
                      "ef_build": w["efb"], "iters": w["iters"], "wall_s": wall,
                      "report": rep}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batched-1m128", choices=sorted(WORKLOADS))
    ap.add_argument("--profile", type=int, default=0,
                    help="run N batched steps inside an NVTX range 'lqg_profile' and exit")
    ap.add_argument("--mode", type=int, default=0, choices=sorted(FIXED_TUNING),
                    help="use this kernel mode (see lqg_tuning) instead of the autotuner's choice")
    ap.add_argument("--build-only", action="store_true",
                    help="build the workload's index (no cache), print the build report, exit")
    ap.add_argument("--ef", type=int, default=0, help="--profile: the ef to search with")
    ap.add_argument("--profile-queries", type=int, default=0,
                    help="--profile: search only the first N queries per step")
    ap.add_argument("--fastscan", action="store_true",
                    help="--profile: run the FastScan/RaBitQ search instead of the SQ8 search")
    ap.add_argument("--prepare", action="store_true",
                    help="build (or assemble) the workload's cached index file and rank-0 "
                         "ground truth, then exit")
    ap.add_argument("--export-shipped", default="",
                    help="PART/NPARTS:DIR - write that part of the cached index's packed "
                         "graph (and metadata, ground truth) under DIR, then exit")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]
    if args.build_only:
        build_only(w, args.workload, int(os.environ.get("LOCAL_RANK", "0")))
        return
    if args.prepare:
        base = gen_data(w, "base")
        path, tb = get_index_file(args.workload, w, base, 0)
        ground_truth(args.workload, w, base, gen_data(w, "query"), 0, 0)
        print(json.dumps({"prepared": path, "build_s": tb}), flush=True)
        return
    if args.export_shipped:
        pn, outdir = args.export_shipped.split(":", 1)
        part, nparts = (int(x) for x in pn.split("/"))
        export_shipped(args.workload, w, part, nparts, outdir)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return
        reference_arm(args, w, args.workload)
        return
    if world > 1:
        import datetime

        import torch

        torch.cuda.set_device(local)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local))
    try:
        if w.get("kind") == "build":
            build_arm(args, w, args.workload, local)
        elif w.get("kind") == "uneven":
            uneven_arm(args, w, args.workload, local)
        elif w.get("kind") == "serving":
            serving_arm(args, w, args.workload, local)
        else:
            gpu_arm(args, w, args.workload, rank, world, local)
    finally:
        if world > 1:
            import torch

            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
