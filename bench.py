"""Benchmark of the spatial-join hot path (filter + LOD refine) on B200.

Workload (one step = one whole join on resident tiles): the within-distance
join at tau = 400 of 200k nuclei (1000 vessels x 200 nuclei, icosphere
nuclei of 1280 triangles, ~20k-triangle branching tube vessels, LODs
20/40/60/80/100, Hausdorff level 2), seeded synthetic tiles in the reference's
RAW .dt format.  The reference publishes no numbers, so vs_baseline is null.

  value        triangle pairs refined per second by the tuned form, inputs
               resident in HBM; the mean over K steps of the device time of the
               whole join call (CUDA events on the library's stream, host work
               between its launches included), L2 flushed between steps,
               max over ranks
  plain        the same join through the plain form (one CTA per voxel pair,
               reference FP32 decision rules): the tuned/plain ratio
  e2e          the same metric through the public C ABI from page-locked host
               tile bytes: both tiles attached (metadata copied), the join
               fetching each LOD's refined voxels from the host bytes, result
               read-back, tiles released; fresh tiles every step (the whole
               upload path is reported beside it)
  roofline     the dominant kernel (tuned refine), FP32 CUDA-core bound
  cpu_baseline the reference's own CPU code (MeshDist, octree; compiled from
               source into oracle/_ref) on a bounded sample of query nuclei,
               all host cores

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = "within-400 join, 1000 vessels x 200 nuclei (200k nuclei), LODs 20-100, hausdorff level 2"
N_VESSELS, NUCLEI_PER_VESSEL, TAU, SEED = 1000, 200, 400.0, 20260002
METRIC = "tri-pairs/s of the within-400 spatial join (filter + LOD refine), tuned form"
F_TRI = 966.0      # FLOPs of one full triangle-pair evaluation (3dpipe_b200/csrc/tridist.cuh)
F_CULL = 14.0      # FLOPs of one bounding-sphere cull test (refine_tuned_kernel)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.f = None

    def __enter__(self):
        try:
            self.f = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed loop starts only once the sampler is producing lines
            t0 = time.time()
            while time.time() - t0 < 5.0 and self.proc.poll() is None:
                self.f.flush()
                if os.fstat(self.f.fileno()).st_size > 0:
                    break
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.f:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.f.seek(0)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Pinned:
    """Page-locks numpy buffers in place (cudaHostRegister) so host->device
    copies of the tiles run at full PCIe/C2C speed."""

    def __init__(self, arrays):
        import torch
        self.rt = torch.cuda.cudart()
        self.ptrs = []
        for a in arrays:
            ptr = a.ctypes.data
            if int(self.rt.cudaHostRegister(ptr, a.nbytes, 0)) == 0:
                self.ptrs.append(ptr)

    def release(self):
        for p in self.ptrs:
            self.rt.cudaHostUnregister(p)
        self.ptrs = []


def make_tiles(rank, ws):
    """Generate the tiles.  One rank: the whole workload.  N ranks: rank 0
    generates the whole nuclei tile and splits the query nuclei with the
    product's partitioner (contiguous ranges of about equal estimated work,
    tdp_raw_partition); every rank then generates the nuclei of its own range
    (the generator places them as in the whole tile) and all vessels, so no
    rank holds more than its share of the query tile.  Returns (nuclei tile,
    vessel tile, first global nucleus id, the split bounds, rank 0's whole
    nuclei tile or None)."""
    pkg = importlib.import_module("3dpipe_b200")
    t = time.time()
    if ws == 1:
        nb, vb = pkg.tdp.gen_tiles(N_VESSELS, NUCLEI_PER_VESSEL, seed=SEED)
        log(f"[rank {rank}] generated {nb.size / 1e9:.2f} + {vb.size / 1e9:.2f} GB in {time.time() - t:.1f}s")
        return nb, vb, 0, [0, N_VESSELS * NUCLEI_PER_VESSEL], None
    import torch.distributed as dist
    whole, box = None, [None]
    if rank == 0:
        whole, vb0 = pkg.tdp.gen_tiles(N_VESSELS, NUCLEI_PER_VESSEL, seed=SEED)
        bounds, work = pkg.shard.partition(whole, vb0, ws, within=TAU)
        box = [bounds.tolist()]
        log(f"[rank 0] split {N_VESSELS * NUCLEI_PER_VESSEL} query nuclei into {ws} ranges {box[0]} "
            f"(estimated voxel pairs {[int(w) for w in work]})")
        del vb0
    dist.broadcast_object_list(box, src=0)
    bounds = box[0]
    b, e = pkg.shard.shard_range(bounds, rank)
    nb, vb = pkg.shard.gen_shard_tiles(b, e, N_VESSELS, NUCLEI_PER_VESSEL, SEED)
    log(f"[rank {rank}] nuclei [{b}, {e}): generated {nb.size / 1e9:.2f} + {vb.size / 1e9:.2f} GB "
        f"in {time.time() - t:.1f}s")
    return nb, vb, b, bounds, whole


def base_config():
    """The workload keys both arms print in `config`."""
    return {"workload": WORKLOAD, "n_nuclei": N_VESSELS * NUCLEI_PER_VESSEL, "n_vessels": N_VESSELS, "tau": TAU,
            "seed": SEED, "query": "within", "lods": [20, 40, 60, 80, 100], "hausdorff_level": 2}


def make_tiles_isolated():
    """Generate the tiles in a child process and read their bytes through a
    pipe, so that the reference arm's own process never loads this
    repository's library."""
    code = ("import sys, importlib; sys.path.insert(0, %r); pkg = importlib.import_module('3dpipe_b200'); "
            "nb, vb = pkg.tdp.gen_tiles(%d, %d, seed=%d); o = sys.stdout.buffer; "
            "o.write(int(nb.size).to_bytes(8, 'little')); o.write(int(vb.size).to_bytes(8, 'little')); "
            "o.write(memoryview(nb)); o.write(memoryview(vb)); o.flush()"
            % (str(ROOT), N_VESSELS, NUCLEI_PER_VESSEL, SEED))
    t = time.time()
    p = subprocess.Popen([sys.executable, "-c", code], stdout=subprocess.PIPE)
    hdr = p.stdout.read(16)
    if len(hdr) != 16:
        p.wait()
        raise SystemExit(f"tile generator exited with {p.returncode}")
    bufs = [np.empty(int.from_bytes(hdr[:8], "little"), np.uint8), np.empty(int.from_bytes(hdr[8:], "little"), np.uint8)]
    for b in bufs:
        mv, off = memoryview(b), 0
        while off < b.size:
            n = p.stdout.readinto(mv[off:off + (1 << 26)])
            if not n:
                raise SystemExit("tile generator pipe closed early")
            off += n
    if p.wait() != 0:
        raise SystemExit(f"tile generator exited with {p.returncode}")
    log(f"[reference] generated {bufs[0].size / 1e9:.2f} + {bufs[1].size / 1e9:.2f} GB in a child process "
        f"in {time.time() - t:.1f}s")
    return bufs[0], bufs[1]


def cpu_reference(nb, vb, steps, warmup, sample_queries, target_s=15.0):
    """The reference's CPU implementation (oracle/_ref) on a bounded sample of
    query nuclei, sized so one run takes about target_s seconds."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_bind import ref_join
    threads = os.cpu_count() or 1
    r = ref_join(nb, vb, False, False, tau=TAU, threads=threads, max_queries=sample_queries)
    if r is None:
        return None
    n_total = N_VESSELS * NUCLEI_PER_VESSEL
    sample = min(sample_queries, n_total)
    sec = max(r[2][0], 1e-3)
    # grow the prefix until one run lasts about target_s (or covers every query)
    while sec < 0.5 * target_s and sample < n_total:
        sample = int(min(n_total, sample * min(8.0, max(2.0, target_s / sec))))
        _, _, st = ref_join(nb, vb, False, False, tau=TAU, threads=threads, max_queries=sample)
        sec = max(st[0], 1e-3)
    vals, last = [], None
    for i in range(warmup + steps):
        _, _, st = ref_join(nb, vb, False, False, tau=TAU, threads=threads, max_queries=sample)
        if i >= warmup:
            vals.append(st[1] / st[0])
        last = st
    return {"value": statistics.median(vals), "unit": "tri-pairs/s", "cores": threads, "kind": "reference",
            "sample": (f"all {n_total} query nuclei (the whole join), " if sample >= n_total else
                       f"first {sample} of {n_total} query nuclei (all their candidate vessels, all LODs), ")
                      + f"median of {steps} run(s) of {last[0]:.1f} s, {last[1]:.3g} tri-pairs each"
                      + ("" if sample >= n_total else
                         f"; join seconds for all nuclei extrapolate linearly to {last[0] * n_total / sample:.0f} s"),
            "seconds_per_sample": last[0], "tri_pairs_per_sample": last[1]}


def check_parity(nb, vb, q, t):
    """The tuned form's within-400 result set against the reference's join
    rules (oracle/_ref: its octree and FP32 MeshDist, all host cores) on the
    whole join; exits when they differ."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_bind import ref_join
    r = ref_join(nb, vb, False, False, tau=TAU, threads=os.cpu_count() or 1)
    if r is None:
        return {"checked": False, "why": "oracle/_ref was not built"}
    got = set(zip(q.tolist(), t.tolist()))
    ref = set(zip(r[0].tolist(), r[1].tolist()))
    out = {"checked": True, "ref_rules_equal": got == ref, "results": len(got), "ref_results": len(ref),
           "only_ours": len(got - ref), "only_ref": len(ref - got), "queries": "all",
           "ref_seconds": r[2][0]}
    log(f"parity within-{TAU:g}: {out}")
    if got != ref:
        print(json.dumps({"parity_failure": out}), file=sys.stderr)
        raise SystemExit("the tuned result set differs from the reference rules' set")
    return out


def check_parity_self_sample(nb, q, t, n_sample):
    """The 10-NN self-join's lists for a stratified sample of query nuclei
    (every n/n_sample-th, from 137) against the reference rules run for
    exactly those queries; exits when they differ."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_bind import ref_join
    n = int(q.max()) + 1 if len(q) else 0
    step = max(1, n // max(1, n_sample))
    sample = np.arange(137 % step, n, step, dtype=np.int32)
    r = ref_join(nb, None, True, True, knn=10, threads=os.cpu_count() or 1, queries=sample)
    if r is None:
        return {"checked": False, "why": "oracle/_ref was not built"}
    sel = np.isin(q, sample)
    got = set(zip(q[sel].tolist(), t[sel].tolist()))
    ref = set(zip(r[0].tolist(), r[1].tolist()))
    out = {"checked": True, "ref_rules_equal": got == ref, "sample_queries": int(len(sample)),
           "sample": f"every {step}th query nucleus from {137 % step}", "results": len(got),
           "ref_results": len(ref), "ref_seconds": r[2][0]}
    log(f"parity 10-NN self-join sample: {out}")
    if got != ref:
        print(json.dumps({"parity_failure": out}), file=sys.stderr)
        raise SystemExit("the 10-NN self-join lists differ from the reference rules' on the sample")
    return out


def run_serving(pkg, ctx, T2, nb, rates, per_rate_cap=600, seconds=3.0, pool_size=48, seed=20260005):
    """Config 5: a served stream of query batches against the resident vessel
    tile.  Requests are contiguous runs of 1-5000 nuclei (log-uniform) of the
    200k-nuclei tile, 60 % kNN with K uniform in 1-50, 40 % within with tau
    uniform in 50-800, Poisson arrivals at each rate for `seconds` (at most
    per_rate_cap requests).  The batching server (tdp_server_*) is compared
    with plain per-request launches (tile upload + tdp_join + free per request,
    one at a time in arrival order) on the same arrival schedule.  Latency =
    arrival to result ready, host clock."""
    import threading
    rng = np.random.default_rng(seed)
    off = pkg.tdp.raw_object_offsets(nb)
    n_total = len(off) - 1
    pool, sizes = [], []
    for _ in range(pool_size):
        n = int(np.clip(np.round(np.exp(rng.uniform(0.0, np.log(5000.0)))), 1, 5000))
        b = int(rng.integers(0, n_total - n + 1))
        pool.append(pkg.tdp.raw_slice(nb, off, b, b + n))
        sizes.append(n)
    pinned = Pinned(pool)

    def schedule(rate):
        n = int(min(per_rate_cap, max(1, round(rate * seconds))))
        t = np.cumsum(rng.exponential(1.0 / rate, n))
        reqs = []
        for k in range(n):
            i = int(rng.integers(0, pool_size))
            if rng.random() < 0.6:
                reqs.append((t[k], i, "nn", int(rng.integers(1, 51)), 0.0))
            else:
                reqs.append((t[k], i, "within", 1, float(rng.uniform(50.0, 800.0))))
        return reqs

    def pct(v, q):
        return float(np.percentile(np.asarray(v), q)) if v else None

    out = []
    for rate in rates:
        reqs = schedule(rate)
        nuclei = sum(sizes[i] for _, i, _, _, _ in reqs)
        # batching server
        with pkg.tdp.Server(ctx, T2) as srv:
            ids = [None] * len(reqs)
            t0 = time.perf_counter()

            def submitter():
                for k, (ta, i, query, K, tau) in enumerate(reqs):
                    dt = t0 + ta - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                    ids[k] = srv.submit(pool[i], query=query, knn=K, within=tau)

            th = threading.Thread(target=submitter)
            th.start()
            th.join()
            lat, batch_sizes, infos = [], [], []
            for rid in ids:
                _, _, _, info = srv.wait(rid)
                lat.append(info["latency_ms"])
                batch_sizes.append(info["batch_requests"])
                infos.append(info)
            wall = time.perf_counter() - t0
            st = srv.stats()
        batched = {"p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "requests_per_s": len(reqs) / wall,
                   "nuclei_per_s": nuclei / wall, "batches": st["batches"],
                   "mean_requests_per_batch": len(reqs) / max(1, st["batches"]),
                   "join_busy_frac": st["busy_ms"] / 1e3 / wall, "h2d_gb_per_s": st["upload_bytes"] / wall / 1e9}
        # the requests behind the tail: the slowest 1 %
        slow = sorted(range(len(reqs)), key=lambda k: -lat[k])[:max(1, len(reqs) // 100)]
        batched["slowest"] = [{"latency_ms": round(lat[k], 2), "nuclei": sizes[reqs[k][1]], "query": reqs[k][2],
                               "knn": reqs[k][3] if reqs[k][2] == "nn" else None,
                               "tau": round(reqs[k][4], 1) if reqs[k][2] == "within" else None,
                               "batch_requests": batch_sizes[k],
                               **{f: round(infos[k][f], 2) for f in ("queue_ms", "join_ms") if f in infos[k]}}
                              for k in slow]
        # plain per-request launches, same schedule
        lat2 = []
        t0 = time.perf_counter()
        for ta, i, query, K, tau in reqs:
            dt = t0 + ta - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            T1 = pkg.tdp.Tile(ctx, pool[i])
            ctx.join(T1, T2, query=query, knn=K, within=tau)
            T1.free()
            lat2.append((time.perf_counter() - (t0 + ta)) * 1e3)
        wall2 = time.perf_counter() - t0
        per_request = {"p50_ms": pct(lat2, 50), "p99_ms": pct(lat2, 99), "requests_per_s": len(reqs) / wall2,
                       "nuclei_per_s": nuclei / wall2}
        log(f"serving rate {rate}/s: {len(reqs)} requests; batched p50 {batched['p50_ms']:.1f} p99 "
            f"{batched['p99_ms']:.1f} ms; per-request p50 {per_request['p50_ms']:.1f} p99 {per_request['p99_ms']:.1f} ms")
        out.append({"rate_per_s": rate, "requests": len(reqs), "nuclei": nuclei, "batched": batched,
                    "per_request": per_request})
    pinned.release()
    return {"workload": "served stream on the resident 1000-vessel tile: requests of 1-5000 nuclei (log-uniform), "
                        "60% kNN k~U[1,50], 40% within tau~U[50,800], Poisson arrivals",
            "pool": f"{pool_size} request tiles sliced from the 200k-nuclei tile (page-locked), reused across arrivals "
                    "with fresh query parameters",
            "latency": "arrival to result ready (host clock); throughput over the whole run including the drain",
            "rates": out}


def run_bounds_prep(pkg, ctx, nb, vb, n_nuclei=20000):
    """GPU preparation of the per-triangle bounds (tdp_tile_compute_bounds) on
    the first n_nuclei objects of the query tile and on the whole vessel tile,
    each on its own resident copy (the joined tiles keep their bounds), beside
    the FP64 CPU restatement of the same rule (oracle/bounds_oracle.cpp, all
    host cores) on a few objects of each."""
    import ctypes
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_bind import oracle
    L = oracle().L
    L.tdo_tile_bounds.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_double)]
    cores = os.cpu_count() or 1
    cpu_nuclei, cpu_vessels = 4 * cores, cores  # a few objects per host core
    offn, offv = pkg.tdp.raw_object_offsets(nb), pkg.tdp.raw_object_offsets(vb)
    n_nuc = min(n_nuclei, len(offn) - 1)
    parts = {"nuclei": (pkg.tdp.raw_slice(nb, offn, 0, n_nuc), pkg.tdp.raw_slice(nb, offn, 0, min(cpu_nuclei, n_nuc))),
             "vessels": (vb, pkg.tdp.raw_slice(vb, offv, 0, min(cpu_vessels, len(offv) - 1)))}
    out = {"workload": f"bounds of the first {n_nuc} nuclei and of all {len(offv) - 1} vessels of the join's tiles "
                       "(LODs 20-80 from each object's LOD-100 surface)"}
    for name, (raw, sample) in parts.items():
        T = pkg.tdp.Tile(ctx, raw)
        ctx.compute_bounds(T)  # untimed first run
        info = ctx.compute_bounds(T)
        T.free()
        smp = np.ascontiguousarray(sample)
        res = np.empty_like(smp)
        ev = ctypes.c_double()
        n_cpu = len(pkg.tdp.raw_object_offsets(smp)) - 1
        t0 = time.perf_counter()
        L.tdo_tile_bounds(smp.ctypes.data, smp.size, res.ctypes.data, 1, cores, ctypes.byref(ev))
        cpu_s = time.perf_counter() - t0
        gpu_rate = info["objects"] / (info["ms"] / 1e3)
        out[name] = {"objects": info["objects"], "triangles": info["triangles"], "gpu_ms": info["ms"],
                     "objects_per_s": gpu_rate, "dist_evals": info["dist_evals"],
                     "dist_evals_per_s": info["dist_evals"] / (info["ms"] / 1e3),
                     "facet_queries": info["facet_queries"], "pieces": info["pieces"],
                     "cpu_objects_per_s": n_cpu / cpu_s, "cpu_cores": cores,
                     "cpu_sample": f"first {n_cpu} {name}, FP64 restatement, one run of {cpu_s:.2f} s",
                     "gpu_over_cpu": gpu_rate / (n_cpu / cpu_s)}
        log(f"bounds {name}: {info['objects']} objects in {info['ms']:.0f} ms on the GPU "
            f"({gpu_rate:.0f}/s), CPU {n_cpu / cpu_s:.1f}/s on {cores} cores")
    return out


def run_lod_prep(pkg, ctx, n_nuclei=20000, n_vessels=100):
    """GPU LOD preparation (tdp_raw_from_meshes: decimation, voxels, RAW writer
    and bounds on the device) of the LOD-100 meshes of the first n_nuclei
    nuclei and n_vessels vessels of the join's generator, beside the CPU
    restatement of the same rule (oracle/lodprep_oracle.cpp on all host cores,
    then the FP64 bound oracle) on a few objects of each; the GPU tile of a
    small sample must equal the CPU one byte for byte."""
    import ctypes
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_bind import oracle
    L = oracle().L
    P = ctypes.c_void_p
    L.tdo_raw_from_meshes.argtypes = [P, P, P, P, ctypes.c_long, ctypes.c_int, P, ctypes.c_size_t,
                                      ctypes.POINTER(ctypes.c_size_t), ctypes.c_int]
    L.tdo_raw_from_meshes.restype = ctypes.c_long
    L.tdo_tile_bounds.argtypes = [P, ctypes.c_size_t, P, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    cores = os.cpu_count() or 1

    def cpu_prep(V, vo, F, fo):
        V, vo, F, fo = (np.ascontiguousarray(x) for x in (V, vo, F, fo))
        n = ctypes.c_size_t()
        args = (V.ctypes.data, vo.ctypes.data, F.ctypes.data, fo.ctypes.data, len(vo) - 1, 100)
        assert L.tdo_raw_from_meshes(*args, None, 0, ctypes.byref(n), cores) == 0
        raw = np.empty(n.value, np.uint8)
        assert L.tdo_raw_from_meshes(*args, raw.ctypes.data, raw.size, ctypes.byref(n), cores) == 0
        out = np.empty_like(raw)
        ev = ctypes.c_double()
        assert L.tdo_tile_bounds(raw.ctypes.data, raw.size, out.ctypes.data, 1, cores, ctypes.byref(ev)) == 0
        return out

    def sub(V, vo, F, fo, k):
        return V[:vo[k]], vo[:k + 1], F[:fo[k]], fo[:k + 1]

    out = {"workload": f"LOD preparation of the LOD-100 meshes of the first {n_nuclei} nuclei and {n_vessels} "
                       "vessels of the join's generator: LODs 80/60/40/20 by half-edge collapse, voxels of ~100 "
                       "facets, RAW bytes, per-triangle bounds"}
    kinds = {"nuclei": pkg.tdp.gen_meshes(N_VESSELS, NUCLEI_PER_VESSEL, seed=SEED, which="nuclei", nuclei_end=n_nuclei),
             "vessels": pkg.tdp.gen_meshes(N_VESSELS, NUCLEI_PER_VESSEL, seed=SEED, which="vessels")}
    kinds["vessels"] = sub(*kinds["vessels"], n_vessels)
    for name, (V, vo, F, fo) in kinds.items():
        k_cpu = 4 * cores if name == "nuclei" else cores
        k_cpu = min(k_cpu, len(vo) - 1)
        small = sub(V, vo, F, fo, min(k_cpu, 8))
        got, _ = ctx.raw_from_meshes(*small)            # untimed first run, checked below
        equal = bool(np.array_equal(np.array(got), cpu_prep(*small)))
        raw, info = ctx.raw_from_meshes(V, vo, F, fo)
        t0 = time.perf_counter()
        cpu_prep(*sub(V, vo, F, fo, k_cpu))
        cpu_s = time.perf_counter() - t0
        n_obj = len(vo) - 1
        gpu_rate = n_obj / (info["total_ms"] / 1e3)
        out[name] = {"objects": n_obj, "facets": int(fo[-1]), "raw_bytes": int(raw.size), "gpu": info,
                     "objects_per_s": gpu_rate, "sample_equal_to_cpu": equal,
                     "cpu_objects_per_s": k_cpu / cpu_s, "cpu_cores": cores,
                     "cpu_sample": f"first {k_cpu} {name}: CPU restatement + FP64 bound oracle, one run of {cpu_s:.2f} s",
                     "gpu_over_cpu": gpu_rate / (k_cpu / cpu_s)}
        log(f"lod prep {name}: {n_obj} objects in {info['total_ms']:.0f} ms (decimate {info['decimate_ms']:.0f}, "
            f"voxels {info['voxel_ms']:.0f}, write {info['write_ms']:.0f}, bounds {info['bounds_ms']:.0f} ms), "
            f"CPU {k_cpu / cpu_s:.1f}/s on {cores} cores, sample equal: {equal}")
        del raw
    return out


def run_out_of_core_stream(a, pkg):
    """Config 4 at its stated size: the 10-NN join of 2M nuclei (10,000 vessels
    x 200) against the 10,000 vessels under a 16 GB device budget.  The 340 GB
    nuclei tile does not fit the host, so it is produced in `ooc_stream` ranges
    of nuclei by a host thread (the generator in place of the reference's CPU
    mesh decoding), at most two ranges in memory; each range is joined by
    tdp_join_chunked against the whole vessel tile while the next one is made.
    Query objects are independent given tile 2, so the ranges' results
    concatenate to the whole join.  Timed end to end: from the first range's
    generation to the last range's results."""
    import queue
    import threading
    import torch
    nv, npv, k = a.ooc_vessels, a.ooc_nuclei_per_vessel, a.ooc_stream
    n = nv * npv
    seed = SEED + 2
    t = time.time()
    _, vb = pkg.tdp.gen_tiles(nv, npv, seed=seed, only="vessels")
    log(f"out-of-core stream: vessel tile {vb.size / 1e9:.1f} GB in {time.time() - t:.0f}s (placement of {n} nuclei included)")
    bounds = [n * i // k for i in range(k + 1)]
    ready = queue.Queue(maxsize=1)
    slots = threading.Semaphore(2)   # nuclei ranges alive at once
    gen_s = [0.0] * k

    def produce():
        for i in range(k):
            slots.acquire()
            t0 = time.perf_counter()
            nb, _ = pkg.tdp.gen_tiles(nv, npv, seed=seed, only="nuclei", nuclei_begin=bounds[i],
                                      nuclei_end=bounds[i + 1])
            gen_s[i] = time.perf_counter() - t0
            ready.put((i, nb))

    budget = int(a.ooc_budget_gb * (1 << 30))
    counts = np.zeros(n, np.int64)
    total, tri, h2d, join_ms, peak, chunks, splits, join_s, nuc_bytes = 0, 0.0, 0.0, 0.0, 0.0, 0, 0, 0.0, 0
    sample = None
    with pkg.Context(0, budget) as ctx:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        th = threading.Thread(target=produce)
        th.start()
        for _ in range(k):
            i, nb = ready.get()
            tj = time.perf_counter()
            q, r, d, info = ctx.join_chunked(nb, vb, a.ooc_chunk, query="nn", knn=10)
            join_s += time.perf_counter() - tj
            nuc_bytes += nb.size
            np.add.at(counts, q.astype(np.int64) + bounds[i], 1)
            total += len(q)
            tri += info["tri_pairs"]
            h2d += info["h2d_bytes"]
            join_ms += info["join_ms"]
            peak = max(peak, info["device_peak_bytes"])
            chunks += info["chunks"]
            splits += info["splits"]
            if i == 0 and not a.no_parity:  # kept for the check after the clock
                qs = np.arange(0, min(len(counts), bounds[1]), max(1, bounds[1] // 100), dtype=np.int32)
                sel = np.isin(q, qs)
                sample = (nb, qs, q[sel].copy(), r[sel].copy())
            del nb, q, r, d
            slots.release()
        th.join()
        wall = time.perf_counter() - t0
    parity = None
    if sample is not None:
        sys.path.insert(0, str(ROOT / "tests"))
        from oracle_bind import ref_join
        nb0, qs, gq, gr = sample
        rr = ref_join(nb0, vb, False, True, knn=10, queries=qs)
        if rr is not None:
            want = set(zip(rr[0].tolist(), rr[1].tolist()))
            got = set(zip(gq.tolist(), gr.tolist()))
            parity = {"checked": True, "ref_rules_equal": want == got, "sample_queries": int(len(qs)),
                      "sample": f"every {max(1, bounds[1] // 100)}th nucleus of the first range", "results": len(got)}
            log(f"out-of-core stream parity: {parity}")
    line = {"metric": "seconds of the out-of-core 10-NN nuclei-vessel join (end to end)", "value": wall,
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"10-NN join, {n} nuclei ({npv} per vessel) x {nv} vessels, LODs 20-100, "
                                   f"device budget {a.ooc_budget_gb:g} GiB, nuclei made in {k} ranges on the host",
                       "tile_bytes": {"nuclei": int(nuc_bytes), "vessels": int(vb.size)},
                       "chunk_objects": a.ooc_chunk, "ranges": k},
            "results": int(total), "every_query_has_k": bool((counts == 10).all()),
            "tri_pairs": tri, "tri_pairs_per_s": tri / wall, "chunks": chunks, "chunk_splits": splits,
            "h2d_gb": h2d / 1e9, "device_join_ms": join_ms, "device_peak_gb": peak / 1e9,
            "join_wall_s": join_s, "generation_s": gen_s, "parity": parity}
    print(json.dumps(line))
    return 0


def run_out_of_core(a):
    """Config 4 scaled to the host: a 10-NN join of nuclei against 10,000
    vessels under a 16 GB device budget, both tiles in host memory (the vessel
    tile alone exceeds the budget), joined in chunks by tdp_join_chunked and
    timed end to end from host bytes to results (one JSON line).  With
    --ooc-stream K the nuclei are made in K ranges while the join runs
    (run_out_of_core_stream), so the stated 2M-nucleus size fits the host."""
    import torch
    pkg = importlib.import_module("3dpipe_b200")
    if a.ooc_stream > 1:
        return run_out_of_core_stream(a, pkg)
    nv, npv = a.ooc_vessels, a.ooc_nuclei_per_vessel
    t = time.time()
    nb, vb = pkg.tdp.gen_tiles(nv, npv, seed=SEED + 2)
    log(f"out-of-core: generated {nb.size / 1e9:.1f} + {vb.size / 1e9:.1f} GB in {time.time() - t:.0f}s")
    budget = int(a.ooc_budget_gb * (1 << 30))
    with pkg.Context(0, budget) as ctx:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        q, r, d, info = ctx.join_chunked(nb, vb, a.ooc_chunk, query="nn", knn=10)
        wall = time.perf_counter() - t0
    n = nv * npv
    line = {"metric": "seconds of the out-of-core 10-NN nuclei-vessel join (end to end)", "value": wall,
            "unit": "s", "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"10-NN join, {n} nuclei ({npv} per vessel) x {nv} vessels, LODs 20-100, "
                                   f"device budget {a.ooc_budget_gb:g} GiB",
                       "tile_bytes": {"nuclei": int(nb.size), "vessels": int(vb.size)},
                       "chunk_objects": a.ooc_chunk},
            "results": int(len(q)), "tri_pairs": info["tri_pairs"], "tri_pairs_per_s": info["tri_pairs"] / wall,
            "chunks": info["chunks"], "chunk_splits": info["splits"], "h2d_gb": info["h2d_bytes"] / 1e9,
            "device_join_ms": info["join_ms"], "device_peak_gb": info["device_peak_bytes"] / 1e9}
    print(json.dumps(line))
    return 0


def run_reference_arm(a):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    ref_so = ROOT / "oracle" / "_ref" / "libtdp_ref.so"
    if not ref_so.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libtdp_ref.so was not built "
                                                               "(needs the reference sources at build time)"}))
        return 0
    nb, vb = make_tiles_isolated()
    # each step a bounded sample, sized so the whole run stays within about 3 minutes
    warm = max(0, min(a.warmup, 1))
    cb = cpu_reference(nb, vb, a.steps, warm, a.cpu_sample, target_s=max(2.0, 150.0 / (a.steps + warm)))
    line = {"metric": METRIC, "value": cb["value"], "unit": "tri-pairs/s", "n_gpus": a.gpus, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": cb["seconds_per_sample"] * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**base_config(), "impl": "reference CPU (MeshDist + octree compiled from source)"},
            "impl": "reference", "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": "tri-pairs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-sample", type=int, default=1500, help="query nuclei in the CPU-baseline sample")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-parity", action="store_true", help="skip the reference-rule result-set checks")
    ap.add_argument("--self-sample", type=int, default=500,
                    help="query nuclei (stratified) whose 10-NN self-join lists are checked against the reference")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--exact-steps", type=int, default=3, help="timed joins with the exact-distance stage")
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream measurement")
    ap.add_argument("--no-self", action="store_true", help="skip the 10-NN self-join measurement")
    ap.add_argument("--no-bounds", action="store_true", help="skip the GPU bound-preparation measurement")
    ap.add_argument("--no-prep", action="store_true", help="skip the GPU LOD-preparation measurement")
    ap.add_argument("--refine-config", type=int, default=-1,
                    help="tuned refine configuration (default: autotuned in the warm-up)")
    ap.add_argument("--out-of-core", action="store_true",
                    help="config 4 instead: the chunked 10-NN join under a device budget (its own JSON line)")
    ap.add_argument("--ooc-vessels", type=int, default=10000)
    ap.add_argument("--ooc-nuclei-per-vessel", type=int, default=50)
    ap.add_argument("--ooc-budget-gb", type=float, default=16.0)
    ap.add_argument("--ooc-chunk", type=int, default=1 << 30, help="max query objects per chunk (the budget cuts them)")
    ap.add_argument("--ooc-stream", type=int, default=1,
                    help="make the nuclei in this many ranges while the join runs (1: the whole tile up front)")
    ap.add_argument("--serve-rates", type=float, nargs="*", default=[200.0, 500.0, 1000.0, 2000.0])
    ap.add_argument("--vessels", type=int, default=None, help="smaller workload for profiling captures")
    ap.add_argument("--nuclei-per-vessel", type=int, default=None)
    a = ap.parse_args()
    global N_VESSELS, NUCLEI_PER_VESSEL, WORKLOAD
    if a.vessels or a.nuclei_per_vessel:
        N_VESSELS = a.vessels or N_VESSELS
        NUCLEI_PER_VESSEL = a.nuclei_per_vessel or NUCLEI_PER_VESSEL
        WORKLOAD = (f"within-400 join, {N_VESSELS} vessels x {NUCLEI_PER_VESSEL} nuclei (reduced, profiling), "
                    "LODs 20-100, hausdorff level 2")
    if a.impl == "reference":
        return run_reference_arm(a)
    if a.out_of_core:
        return run_out_of_core(a)

    import torch
    import torch.distributed as dist
    ws, rank, local = dist_env()
    if ws > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    pkg = importlib.import_module("3dpipe_b200")
    nb, vb, first, bounds, whole = make_tiles(rank, ws)
    t = time.time()
    pinned = Pinned([nb, vb])
    log(f"[rank {rank}] page-locked {len(pinned.ptrs)} tile buffers in {time.time() - t:.1f}s")

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def allmax(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def allsum(x):
        if ws == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    out = {}
    with pkg.Context(local) as ctx:
        fp32_peak = ctx.fp32_peak()
        t = time.time()
        T1, T2 = pkg.tdp.Tile(ctx, nb), pkg.tdp.Tile(ctx, vb)
        log(f"[rank {rank}] tiles resident in {time.time() - t:.1f}s, {ctx.memory()[0] / 1e9:.1f} GB on device")
        # pick the tuned refine kernel's configuration on this join (untimed),
        # or take the one given on the command line
        if a.refine_config >= 0:
            ctx.set_refine_config(a.refine_config)
            best_cfg, cfg_ms = a.refine_config, []
        else:
            best_cfg, cfg_ms = ctx.autotune(T1, T2, query="within", within=TAU)
        cfg_defs = pkg.tdp.refine_configs()
        cfg_by_lod = ctx.refine_configs_by_lod()
        log(f"[rank {rank}] autotune: refine ms per configuration {[round(m, 3) for m in cfg_ms]} -> {best_cfg}, "
            f"per LOD {cfg_by_lod}")
        # the two forms must agree before anything is timed
        qa, ra, _ = ctx.join(T1, T2, query="within", within=TAU, form=pkg.FORM_PLAIN)
        qb, rb, _ = ctx.join(T1, T2, query="within", within=TAU, form=pkg.FORM_TUNED)
        if not (np.array_equal(qa, qb) and np.array_equal(ra, rb)):
            raise SystemExit("plain and tuned forms returned different result sets")
        n_results = len(qb)
        # and the reference's own join rules (its octree and FP32 MeshDist,
        # compiled from source, all host cores) must give the same set
        parity = {"within400": None, "knn10_self_sample": None}
        if ws == 1 and not a.no_parity:
            parity["within400"] = check_parity(nb, vb, qb, rb)
        elif ws > 1:
            # every rank's result, ids mapped to global ones, gathered on rank
            # 0; there the union must equal the reference rules' set of the
            # whole join (after the timed steps: the check takes host cores)
            merged = pkg.shard.gather_results(pkg.shard.to_global(qb, first), rb, np.zeros(len(qb)), dst=0)

        # Every join launches on the context's stream; the step events are
        # recorded on that same stream.  Between steps a 256 MiB buffer (twice
        # L2) is rewritten on the stream, outside the step's events, so no
        # step starts with the previous step's lines in L2.
        stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=torch.device("cuda", local))
        flush_buf = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

        def timed(form, steps, warmup):
            for _ in range(warmup):
                ctx.join(T1, T2, query="within", within=TAU, form=form)
            barrier()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(steps)]
            sts = []
            for e0, e1 in evs:
                with torch.cuda.stream(stream):
                    flush_buf.fill_(len(sts) & 0xff)
                    e0.record(stream)
                ctx.join(T1, T2, query="within", within=TAU, form=form)
                with torch.cuda.stream(stream):
                    e1.record(stream)
                sts.append(ctx.stats())
            barrier()
            ms = sum(e0.elapsed_time(e1) for e0, e1 in evs) / steps
            agg = {k: sum(s[k] for s in sts) / steps for k in ("refine_ms", "full_evals", "tri_pairs")}
            launches = sum(s["kernel_launches"] for s in sts)
            return ms, sts[-1], agg, launches

        with ClockSampler(local) as clk:
            ms_t, st_t, agg_t, launches_t = timed(pkg.FORM_TUNED, a.steps, a.warmup)
        clocks = clk.summary()
        ms_p, st_p, agg_p, _ = timed(pkg.FORM_PLAIN, max(3, a.steps // 4), 1)

        step_ms = allmax(ms_t)
        tri = allsum(st_t["tri_pairs"])
        value = tri / (step_ms / 1e3)
        plain_ms = allmax(ms_p)
        plain_value = allsum(st_p["tri_pairs"]) / (plain_ms / 1e3)
        refine_ms = agg_t["refine_ms"]
        launches_refine = max(1, st_t["refine_launches"])
        flops = agg_t["full_evals"] * F_TRI + agg_t["tri_pairs"] * F_CULL
        achieved = flops / (refine_ms / 1e3) / 1e12

        # config 3: the 10-NN self-join over the same 200k nuclei (tuned form;
        # one run to build the grids, one measured by the library's events)
        knn_self = None
        if not a.no_self and ws == 1:
            ctx.join(T1, None, query="nn", knn=10, form=pkg.FORM_TUNED)
            qs, ts, _ = ctx.join(T1, None, query="nn", knn=10, form=pkg.FORM_TUNED)
            st_s = ctx.stats()
            if not a.no_parity:
                parity["knn10_self_sample"] = check_parity_self_sample(nb, qs, ts, a.self_sample)
            knn_self = {"workload": f"10-NN self-join over the {N_VESSELS * NUCLEI_PER_VESSEL} nuclei, LODs 20-100",
                        "join_ms": st_s["total_ms"], "tri_pairs": st_s["tri_pairs"],
                        "tri_pairs_per_s": st_s["tri_pairs"] / (st_s["total_ms"] / 1e3),
                        "refine_ms": st_s["refine_ms"], "voxel_pairs_refined": st_s["refine_items"],
                        "results": int(len(qs)), "recheck_pairs": st_s["recheck_pairs"]}
            log(f"[rank {rank}] knn self-join: {st_s['total_ms']:.0f} ms, "
                f"{knn_self['tri_pairs_per_s'] / 1e9:.1f} G tri-pairs/s")

        # the join with the exact-distance stage (every result's LOD-100
        # distance in FP64): one warm-up, then the median of 3 joins, device
        # time by the library's events; the FP32 refine's error against FP64
        exact = None
        if a.exact_steps > 0:
            ctx.join(T1, T2, query="within", within=TAU, form=pkg.FORM_TUNED, exact_distances=True)
            xs = []
            for _ in range(a.exact_steps):
                ctx.join(T1, T2, query="within", within=TAU, form=pkg.FORM_TUNED, exact_distances=True)
                xs.append(ctx.stats())
            xs.sort(key=lambda st: st["total_ms"])
            st_x = xs[len(xs) // 2]
            exact = {"join_ms": st_x["total_ms"], "exact_ms": st_x["exact_ms"],
                     "over_join_without": st_x["total_ms"] / step_ms if step_ms else None,
                     "phase_ms": dict(zip(("upper_bounds", "candidates", "fp32_pass", "fp64_pass"),
                                          st_x["exact_phase_ms"])),
                     "voxel_pairs_fp32": st_x["exact_items"], "voxel_pairs_fp64": st_x["exact_f64_items"],
                     "fp32_full_evals": st_x["exact_full_evals"], "fp32_max_rel_err": st_x["fp32_max_rel_err"],
                     "fp32_items_dropped": st_x["exact_dropped_items"],
                     "fp32_items_below_preset": st_x["exact_below_items"],
                     "steps": a.exact_steps, "note": "median of the timed joins; resident tiles"}

        # end to end through the C ABI from the page-locked host tile bytes:
        # attach both tiles (voxel metadata up), join (each LOD fetches the
        # triangles of the voxels it refines from the host bytes), result
        # read-back, tile release -- between two events on the context's
        # stream, every step on freshly attached tiles.  The same with whole
        # uploads (every byte of both tiles copied and unpacked) is measured
        # once beside it.
        def e2e_step_run(attach):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h0 = time.perf_counter()
            U1, U2 = pkg.tdp.Tile(ctx, nb, attach=attach), pkg.tdp.Tile(ctx, vb, attach=attach)
            h1 = time.perf_counter()
            q, r, d = ctx.join(U1, U2, query="within", within=TAU, form=pkg.FORM_TUNED)
            h2 = time.perf_counter()
            sj = ctx.stats()
            fetched = sj["fetch_bytes"]
            i1, i2 = U1.info(), U2.info()
            h2d_b = i1["h2d_bytes"] + i2["h2d_bytes"] + int(fetched)
            U1.free(); U2.free()
            e1.record(stream)
            e1.synchronize()
            h3 = time.perf_counter()
            return (e0.elapsed_time(e1), h2d_b, q.nbytes + r.nbytes + d.nbytes,
                    {"tiles_ms": 1e3 * (h1 - h0), "parse_ms": i1["parse_ms"] + i2["parse_ms"],
                     "alloc_ms": i1["alloc_ms"] + i2["alloc_ms"], "meta_ms": i1["meta_ms"] + i2["meta_ms"],
                     "load_ms": i1["load_ms"] + i2["load_ms"], "join_ms": 1e3 * (h2 - h1),
                     "fetch_bytes": fetched, "release_ms": 1e3 * (h3 - h2),
                     "join_device": {k: sj[k] for k in ("total_ms", "candidates_ms", "filter_ms", "lod_ms", "refine_ms",
                                                        "host_syncs", "lod_graph")}})

        e2e_ms, h2d, d2h, e2e_parts = [], 0, 0, None
        for i in range(a.e2e_steps + 1 if a.e2e_steps > 0 else 0):
            barrier()
            ms, h2d, d2h, e2e_parts = e2e_step_run(True)
            if i > 0:
                e2e_ms.append(ms)
        e2e_step = allmax(statistics.median(e2e_ms)) if e2e_ms else float("nan")
        e2e_value = tri / (e2e_step / 1e3) if e2e_ms else None
        # the same end to end with the exact-distance stage (one step)
        e2e_exact = None
        if a.e2e_steps > 0 and a.exact_steps > 0:
            barrier()
            x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x0.record(stream)
            U1, U2 = pkg.tdp.Tile(ctx, nb, attach=True), pkg.tdp.Tile(ctx, vb, attach=True)
            qx, rx, dx = ctx.join(U1, U2, query="within", within=TAU, form=pkg.FORM_TUNED, exact_distances=True)
            fx = ctx.stats()["fetch_bytes"]
            hx = U1.info()["h2d_bytes"] + U2.info()["h2d_bytes"] + int(fx)
            U1.free(); U2.free()
            x1.record(stream)
            x1.synchronize()
            e2e_exact = {"ms_per_step": allmax(x0.elapsed_time(x1)), "h2d_bytes_per_step": int(hx),
                         "d2h_bytes_per_step": int(qx.nbytes + rx.nbytes + dx.nbytes), "results": int(len(qx)),
                         "note": "attach x2 + join with FP64 exact distances + read-back + release, one step"}
        e2e_upload = None
        if a.e2e_steps > 0:
            barrier()
            ms_u, h2d_u, _, parts_u = e2e_step_run(False)
            e2e_upload = {"value": tri / (allmax(ms_u) / 1e3), "unit": "tri-pairs/s", "ms_per_step": allmax(ms_u),
                          "h2d_bytes_per_step": int(h2d_u), "host_ms": parts_u,
                          "note": "tiles uploaded whole (every LOD of every object copied and unpacked), one step"}

        serving = None
        if not a.no_serve and ws == 1:
            T1.free()  # the serving arenas replace the resident query tile
            serving = run_serving(pkg, ctx, T2, nb, a.serve_rates)
        bounds_prep = None
        if not a.no_bounds and ws == 1:
            T1.free()
            T2.free()
            bounds_prep = run_bounds_prep(pkg, ctx, nb, vb)
        lod_prep = None
        if not a.no_prep and ws == 1:
            lod_prep = run_lod_prep(pkg, ctx)
        del flush_buf

    pinned.release()
    if ws > 1 and rank == 0 and not a.no_parity:
        gq, gt, _ = merged
        parity["within400"] = check_parity(whole, vb, gq, gt)
        parity["within400"]["shards"] = bounds
    if ws > 1:
        n_results = len(merged[0]) if rank == 0 else n_results
    cpu = None
    if rank == 0 and ws == 1 and not a.no_cpu:
        cpu = cpu_reference(nb, vb, 3, 0, a.cpu_sample, target_s=5.0)
    # DRAM bytes per refine launch from the committed ncu capture of this workload
    traffic = None
    prof = ROOT / "profiles" / "refine_within400.md"
    if prof.exists():
        for ln in prof.read_text().splitlines():
            if ln.startswith("traffic_bytes_per_launch:"):
                try:
                    traffic = float(ln.split(":", 1)[1])
                except ValueError:
                    traffic = None
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "tri-pairs/s", "n_gpus": ws, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {**base_config(), "form": "tuned", "results": n_results,
                       "join_seconds": step_ms / 1e3, "tri_pairs_per_join": tri,
                       "refine_ms": refine_ms, "filter_ms": st_t["filter_ms"],
                       "l2": "L2 flushed between timed steps (256 MiB rewrite on the join stream, outside the step events)",
                       "parallelism": f"{ws} GPU(s)" + ("" if ws == 1 else
                                       ", query nuclei split into contiguous ranges of equal estimated work "
                                       "(tdp_raw_partition), results gathered on rank 0"),
                       "refine_config": {"chunk_a": cfg_defs[best_cfg][0], "ctas_per_sm": cfg_defs[best_cfg][1],
                                         "autotune_refine_ms": [round(m, 4) for m in cfg_ms],
                                         "by_lod": {str(k): {"config": v, "chunk_a": cfg_defs[v][0],
                                                             "ctas_per_sm": cfg_defs[v][1]}
                                                    for k, v in cfg_by_lod.items()}}},
            "plain": {"value": plain_value, "unit": "tri-pairs/s", "ms_per_step": plain_ms,
                      "tuned_over_plain": value / plain_value if plain_value else None},
            "e2e": {"value": e2e_value, "unit": "tri-pairs/s", "ms_per_step": e2e_step,
                    "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "path": "tdp_tile_attach x2 (page-locked host tiles, 36.8 GB) + tdp_join (per-LOD fetch of the "
                            "voxels refined) + result read-back + tdp_tile_free, fresh tiles every step",
                    "host_ms": e2e_parts, "upload_path": e2e_upload, "exact": e2e_exact},
            "parity": parity,
            "exact_distances": exact,
            "serving": serving,
            "bounds_prep": bounds_prep,
            "lod_prep": lod_prep,
            "knn_self_join": knn_self,
            "gpu_launches": int(launches_t),
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved / fp32_peak if fp32_peak else None, "traffic": traffic,
                         "traffic_source": "DRAM read+write bytes per launch: ncu capture of the 20k-nuclei case, "
                                           "scaled by the refined voxel pairs (profiles/refine_within400.md)",
                         "kernel": "refine_lazy_kernel" if cfg_by_lod[100] >= 3 else "refine_tuned_kernel",
                         "peak_source": "measured FP32 FMA probe (tdp_fp32_peak); MEASURED_PEAKS.json has no CUDA-core FP32 figure",
                         "work": f"full evals x {F_TRI:.0f} + culled pairs x {F_CULL:.0f} FLOPs",
                         "tri_pair_equivalent": {
                             "achieved": agg_t["tri_pairs"] * F_TRI / (refine_ms / 1e3) / 1e12,
                             "frac": (agg_t["tri_pairs"] * F_TRI / (refine_ms / 1e3) / 1e12) / fp32_peak
                             if fp32_peak else None,
                             "note": "every triangle pair of every refined voxel pair counted at F_TRI; above 1.0 "
                                     "because the tuned form proves most pairs irrelevant with a ~14-FLOP bound"},
                         "launches_per_step": launches_refine},
            "clocks": clocks,
            "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")} if cpu else None,
            "stats": {k: st_t[k] for k in ("full_evals", "refine_items", "recheck_pairs", "filter_pairs",
                                           "filter_voxel_pairs", "kernel_launches", "candidates_ms", "lod_ms",
                                           "host_syncs", "total_ms")},
        }
        print(json.dumps(line))
    if ws > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
