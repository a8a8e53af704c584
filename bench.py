"""Benchmark of the UMAP hot path on B200: end-to-end seconds and SGD edge-updates/s.

Workload (default): 1,000,000 observations x 50 dims, float32 Gaussian mixture
of 100 clusters (centres N(0, 25 I), within-cluster sd 1, Dirichlet(1)
weights), exact kNN with k = 15, 2-d output, 200 epochs, default Options
otherwise.  Seeded synthetic data (no public dataset is named).

One step = umappp's initialize(data, builder, ...) + Status::run() on the
whole data set: device kNN, similarities, fuzzy union, initial layout,
schedule and 200 SGD epochs.

  value       seconds per step with the data already in HBM (device pointers
              passed to the C ABI); time on the device with CUDA events around
              the step, max over ranks.
  e2e         the same through the public API with pageable->pinned host
              buffers: the H2D copy of the data and the D2H copy of the
              embedding are inside the timed region.
  --impl reference   times the reference (libscran/umappp headers compiled in
              oracle/_ref) on the host cores on a bounded sample and scales it
              to the full workload (see cpu_sample()).

Launch: python bench.py [--gpus N --steps K --warmup W]; for N > 1 under
torchrun, each rank runs an independent replica (UMAP's SGD has no exchange
step), scaling "weak".
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

CONFIGS = {
    # name: (n, dim, clusters, centre_sd, weights, k, epochs)
    "mixture_1m": (1_000_000, 50, 100, 5.0, "dirichlet", 15, 200),
    "mixture_100k": (100_000, 50, 20, 4.0, "equal", 15, 500),
    "small_2k": (2_000, 10, 1, 0.0, "equal", 15, 500),
}
METRIC = "end-to-end s & SGD edge-updates/s, 1M pts; FP32/batched vs plain at equal trust"
# DRAM bytes (read + write) per launch of the dominant kernels, from ncu
# captures summarised in profiles/traffic.json (each entry names the capture
# it comes from and how it was scaled to the workload).
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")
# Batched workload: 64 independent instances, sizes log-uniform in [500, 50000],
# 30 dims, float32 5-cluster mixtures, k = 15, 200 epochs.
BATCH = {"instances": 64, "min": 500, "max": 50_000, "dim": 30, "clusters": 5, "k": 15, "epochs": 200}


def make_data(cfg: str, seed: int = 20241203) -> np.ndarray:
    n, dim, nc, sd, weights, _, _ = CONFIGS[cfg]
    rng = np.random.default_rng(seed)
    centres = rng.normal(0.0, sd, size=(nc, dim)).astype(np.float32)
    p = rng.dirichlet(np.ones(nc)) if weights == "dirichlet" else np.full(nc, 1.0 / nc)
    labels = rng.choice(nc, size=n, p=p)
    out = rng.standard_normal(size=(n, dim), dtype=np.float32)
    out += centres[labels]
    return out


def load_traffic(config: str, kernel: str):
    """(bytes per launch, source note) of a kernel at a workload, or (None, None)."""
    try:
        with open(TRAFFIC_FILE) as f:
            e = json.load(f)[config][kernel]
        return float(e["bytes_per_launch"]), e["source"]
    except (OSError, KeyError, ValueError, TypeError):
        return None, None


def l2_random_access_peaks(U) -> dict:
    """Measured rates of uniformly random float2 loads and atomic adds over a
    10^6-point (8 MB, L2-resident) array: the ceiling of the SGD epochs,
    whose accesses are of that kind (umapb_measure_random_access)."""
    import ctypes

    out = {}
    for mode, name in ((0, "gather_per_s"), (1, "atomic_add_per_s")):
        r = ctypes.c_double()
        U._lib.check(U.lib().umapb_measure_random_access(1_000_000, 400_000_000, mode, 5, ctypes.byref(r)))
        out[name] = r.value
    return out


def sgd_roofline(nnz: int, epochs: int, firing: float, negs: float, sgd_ms: float, peaks: dict, l2: dict,
                 traffic, traffic_src) -> dict:
    """Roofline of the SGD epochs (one launch of sgd_rows_2d_f32 per epoch).
    Against HBM: the algorithmic bytes of the schedule and the layout,
    4 nnz + 56 F + 8 N_neg per epoch (F firing edges, N_neg negative samples,
    exact counts from the schedule), over the SGD stage's CUDA-event time,
    i.e. per launch over the average launch.  Against L2 (frac_l2): the
    epochs' accesses are random 8-byte loads and atomic adds that hit L2 (the
    8 MB embedding stays there) -- per firing edge the head is read and its
    move added, the tail read and moved; per negative sample one read -- and
    their ceiling is the measured rate of such loads and atomic adds, taken in
    proportion: frac_l2 = the time those accesses take at the measured rates
    over the stage time."""
    sgd_s = sgd_ms * 1e-3
    sgd_bytes = 4.0 * nnz * epochs + 56.0 * firing + 8.0 * negs
    sgd_gbs = sgd_bytes / sgd_s / 1e9
    loads, adds = 2.0 * firing + negs, 2.0 * firing
    l2_floor_s = loads / l2["gather_per_s"] + adds / l2["atomic_add_per_s"]
    return {"bound": "hbm", "kernel": "sgd_rows_2d_f32",
            "achieved": round(sgd_gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
            "frac": round(sgd_gbs / peaks["hbm_gbs"], 4), "peak_source": peaks["source"],
            "traffic": traffic, "traffic_unit": "DRAM bytes per epoch launch", "traffic_source": traffic_src,
            "algorithmic_bytes_per_launch": round(sgd_bytes / max(epochs, 1)),
            "time_ms": round(sgd_ms, 3),
            "frac_l2": round(l2_floor_s / sgd_s, 4), "achieved_l2": round((loads + adds) / sgd_s / 1e9, 2),
            "peak_l2": round((loads + adds) / l2_floor_s / 1e9, 2), "unit_l2": "G random L2 accesses/s",
            "peak_l2_source": "measured in this run (umapb_measure_random_access: loads "
                              f"{l2['gather_per_s'] / 1e9:.1f} G/s, atomic adds {l2['atomic_add_per_s'] / 1e9:.1f} G/s)",
            "note": "achieved = 4 nnz + 56 F + 8 N_neg bytes per epoch over the SGD stage time (all epochs); "
                    "the epochs are bound by the latency of each row's chain of L2 accesses, so frac_l2 (the "
                    "4 F + N_neg random accesses at the measured random-access rates over the stage time) is "
                    "the fraction of the ceiling that binds"}


def stage_rooflines(n: int, k: int, nnz: int, stages: dict, peaks: dict, float_bytes: int = 4) -> dict:
    """HBM fractions of the two small graph stages by their algorithmic bytes:
    similarities n k (4 read + 4 write) + 16 n (rho and sigma in FP64);
    union n k 8 read (index and weight) + nnz 8 + (n + 1) 8 written (the CSR
    out; its sort passes are not counted).  nnz is the stored edges after the
    epochs filter, within 0.1 % of the union's output at the benchmark sizes."""
    out = {}
    for name, nbytes in (("similarities", n * k * (2 * float_bytes) + 16 * n),
                         ("union", n * k * (4 + float_bytes) + nnz * (4 + float_bytes) + (n + 1) * 8)):
        ms = float(stages.get(name, 0.0))
        gbs = nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0
        out[name] = {"bound": "hbm", "achieved": round(gbs, 1), "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": round(gbs / peaks["hbm_gbs"], 4), "algorithmic_bytes": int(nbytes),
                     "time_ms": round(ms, 3)}
    return out


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": d["hbm_gbs"], "bf16_tflops": d["bf16_tflops"], "source": "measured"}
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region
    (raw samples kept in $UMAPB_CLOCKS_DIR/clocks_rank<i>.csv when that is set)."""

    def __init__(self, index: int):
        self.proc = None
        out_dir = os.environ.get("UMAPB_CLOCKS_DIR")
        self.path = (os.path.join(out_dir, f"clocks_rank{index}.csv") if out_dir and os.path.isdir(out_dir)
                     else f"/tmp/umapb_clocks_{os.getpid()}.csv")
        self.index = index

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,"
                 "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.f.close()
        except Exception:
            pass

    def summary(self) -> dict:
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            rows = []
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(name)
            except Exception:
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(value: float, world: int, device=None) -> float:
    """The largest of the ranks' values; every rank calls it (one rank: the value)."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------ our arm ---

def run_ours(args, rank: int, world: int) -> dict | None:
    import torch
    import umappp_b200 as U

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    n, dim, _, _, _, k, epochs = CONFIGS[args.config]
    X = make_data(args.config, seed=20241203 + rank)
    opt = U.Options(num_neighbors=k, num_epochs=epochs)

    d_data = torch.from_numpy(X).to(dev)
    d_emb = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    h_data = torch.from_numpy(X).pin_memory()
    h_emb = torch.zeros((n, 2), dtype=torch.float32).pin_memory()

    def step_device():
        st = U.initialize_from_data(d_data, 2, d_emb, opt)
        st.run(d_emb)
        return st

    def step_host():
        st = U.initialize_from_data(h_data.numpy(), 2, h_emb.numpy(), opt)
        st.run(h_emb.numpy())
        return st

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed(fn, steps):
        barrier()
        l0 = U.lib().umapb_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        last = None
        for _ in range(steps):
            last = None   # release the previous step's state before the next step allocates its own
            last = fn()
        e1.record()
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
        return ms, last, U.lib().umapb_launch_count() - l0

    for _ in range(args.warmup):
        step_device()
    with ClockSampler(dev.index) as clk:
        ms, st, launches = timed(step_device, args.steps)
    clocks = clk.summary()
    stages = st.stage_ms()
    counts = st.schedule_counts()
    firing = int(counts[:, 0].sum())
    negs = int(counts[:, 1].sum())
    nnz = st.num_edges()
    sgd_ms = stages["sgd"]
    del st
    # the last timed step's tensor-core kNN: pruned work and kernel time (CUDA events)
    tile_pairs = int(U.lib().umapb_knn_last_tile_pairs())
    knn_kernel_ms = float(U.lib().umapb_knn_last_kernel_ms())
    for _ in range(max(1, args.warmup // 2)):
        step_host()
    e2e_ms, _, _ = timed(step_host, args.steps)

    peaks = load_peaks()
    l2 = l2_random_access_peaks(U)
    traffic_sgd, traffic_sgd_src = load_traffic(args.config, "sgd_rows_2d_f32")
    roof_sgd = sgd_roofline(nnz, epochs, firing, negs, sgd_ms, peaks, l2, traffic_sgd, traffic_sgd_src)
    # kNN roofline: the distances the pruned search computes (128 x 128 per tile pair,
    # 2*dim FLOP each, the FP32 GEMM count) over the kernel's device time
    knn_flops = tile_pairs * 128.0 * 128.0 * 2.0 * dim
    knn_tflops = knn_flops / (knn_kernel_ms * 1e-3) / 1e12 if knn_kernel_ms > 0 else 0.0
    traffic_knn, traffic_knn_src = load_traffic(args.config, "knn_tc16_kernel")
    roof_knn = {"bound": "tensor", "kernel": "knn_tc16_kernel", "achieved": round(knn_tflops, 2),
                "peak": peaks["bf16_tflops"], "unit": "TFLOP/s", "frac": round(knn_tflops / peaks["bf16_tflops"], 4),
                "traffic": traffic_knn, "traffic_unit": "DRAM bytes per launch", "traffic_source": traffic_knn_src,
                "peak_source": peaks["source"], "time_ms": round(knn_kernel_ms, 3),
                "note": "2*dim FLOP per computed (query, reference) pair over the kernel's CUDA-event time; "
                        "peak = measured dense BF16 (FP16 runs at the same rate); the 3-product FP16 split "
                        "and the K padding (dim+1 -> 64) make the issued tensor work 3*64/dim times this",
                "tile_pairs": tile_pairs, "tile_pairs_brute_force": ((n + 127) // 128) ** 2}
    dominant = roof_knn if knn_kernel_ms >= sgd_ms else roof_sgd
    out = {
        "metric": METRIC, "value": round(ms / 1e3, 4), "unit": "s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms, 3), "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian mixture)",
        "config": {"workload": f"{args.config}: n={n} dim={dim} k={k} out_dim=2 epochs={epochs}",
                   "l2": "inputs (200 MB data) larger than L2", "parallelism": f"replicas x{world}"},
        "sgd_edge_updates_per_s": round(firing / (sgd_ms * 1e-3), 1),
        "stage_ms": {k_: round(v, 3) for k_, v in stages.items()},
        "roofline": dominant,
        "roofline_knn": roof_knn,
        "roofline_sgd": roof_sgd,
        "roofline_stages": stage_rooflines(n, k, nnz, stages, peaks),
        "e2e": {"value": round(e2e_ms / 1e3, 4), "unit": "s", "h2d_bytes_per_step": int(n * dim * 4 + n * 2 * 4),
                "d2h_bytes_per_step": int(2 * n * 2 * 4)},
        "gpu_launches": int(launches // max(args.steps, 1)),
        "clocks": clocks,
        "schedule": {"nnz": int(nnz), "firing_edges": firing, "negative_samples": negs},
    }
    return out


def make_batch(seed: int = 20241203):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(BATCH["min"]), np.log(BATCH["max"]), size=BATCH["instances"])).astype(np.int32)
    parts = []
    for m in sizes:
        centres = rng.normal(0.0, 5.0, size=(BATCH["clusters"], BATCH["dim"])).astype(np.float32)
        labels = rng.choice(BATCH["clusters"], size=int(m))
        parts.append(centres[labels] + rng.standard_normal(size=(int(m), BATCH["dim"]), dtype=np.float32))
    return sizes, np.ascontiguousarray(np.concatenate(parts))


def run_batch(args, rank: int, world: int) -> dict | None:
    """64 instances in one umapb_batch_run call against 64 plain
    initialize_from_data + run calls, device-resident inputs for both."""
    import torch
    import umappp_b200 as U

    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sizes, X = make_batch(20241203 + rank)
    n = int(sizes.sum())
    opt = U.Options(num_neighbors=BATCH["k"], num_epochs=BATCH["epochs"])
    d_data = torch.from_numpy(X).to(dev)
    d_emb = torch.zeros((n, 2), dtype=torch.float32, device=dev)
    offs = np.concatenate([[0], np.cumsum(sizes)])
    views = [(d_data[offs[i]:offs[i + 1]], d_emb[offs[i]:offs[i + 1]]) for i in range(len(sizes))]

    def batched():
        return U.batch_run(d_data, sizes, 2, d_emb, opt)

    def sequential():
        for xd, yd in views:
            st = U.initialize_from_data(xd, 2, yd, opt)
            st.run(yd)

    def timed(fn, steps):
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        l0 = U.lib().umapb_launch_count()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        last = None
        for _ in range(steps):
            last = fn()
        e1.record()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps, world, dev)
        return ms, last, (U.lib().umapb_launch_count() - l0) // max(steps, 1)

    for _ in range(args.warmup):
        batched()
    with ClockSampler(dev.index) as clk:
        ms, stages, launches = timed(batched, args.steps)
    sequential()
    seq_ms, _, seq_launches = timed(sequential, 1)
    return {"metric": "batched UMAP: 64 instances, seconds per batch", "value": round(ms / 1e3, 4), "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Gaussian mixtures)",
            "config": {"workload": f"batch64: {len(sizes)} instances, sizes {int(sizes.min())}..{int(sizes.max())} "
                                   f"(total {n}), dim={BATCH['dim']} k={BATCH['k']} epochs={BATCH['epochs']}"},
            "sequential_plain_s": round(seq_ms / 1e3, 4), "speedup_vs_sequential": round(seq_ms / ms, 2),
            "stage_ms": {k_: round(v, 3) for k_, v in stages.items()}, "gpu_launches": int(launches),
            "sequential_gpu_launches": int(seq_launches), "clocks": clk.summary()}


# --------------------------------------------------- reference on CPU ---

def cpu_sample(cfg: str, budget_queries: int = 1000, sub_n: int = 50_000, sgd_epochs: int = 10) -> dict:
    """Times the reference (oracle/_ref) on the host cores and scales it to the full workload:
    - kNN: the stand-in exact brute force on the full data for 'budget_queries'
      queries, scaled by n / queries (the cost is linear in queries);
    - similarities, union, initial layout, schedule: the reference's stages on a
      'sub_n'-point sample of the same mixture (its own exact kNN graph), scaled
      by n / sub_n (each is linear in the number of edges);
    - SGD: the first 'sgd_epochs' epochs of optimize_layout_parallel on that
      sample, scaled by (epochs / sgd_epochs) * (n / sub_n)."""
    import ctypes

    import oracle

    R = oracle.ref()
    R.ref_pipeline_timed_f32.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    n, dim, _, _, _, k, epochs = CONFIGS[cfg]
    cores = os.cpu_count() or 1
    X = make_data(cfg)
    q = min(budget_queries, n)
    t0 = time.perf_counter()
    oracle.ref_knn(X, k, qstart=0, qcount=q, nthreads=cores)
    t_knn = (time.perf_counter() - t0) * n / q
    m = min(sub_n, n)
    rng = np.random.default_rng(7)
    S = np.ascontiguousarray(X[rng.choice(n, size=m, replace=False)])
    emb = np.zeros((m, 2), dtype=np.float32)
    secs = np.zeros(6, dtype=np.float64)
    e_s = min(sgd_epochs, epochs)
    R.ref_pipeline_timed_f32(dim, m, S.ctypes.data, k, epochs, e_s, cores, emb.ctypes.data, secs.ctypes.data)
    scale = n / m
    stages = {"knn": t_knn, "similarities": secs[1] * scale, "union": secs[2] * scale, "init": secs[3] * scale,
              "epochs": secs[4] * scale, "sgd": secs[5] * scale * epochs / e_s}
    total = sum(stages.values())
    return {"value": round(total, 2), "unit": "s", "cores": cores, "kind": "reference",
            "stages_s": {k_: round(v, 2) for k_, v in stages.items()},
            "sample": f"kNN: {q} queries over all {n} points x{n // q}; other stages: {m}-point sample x{scale:g}; "
                      f"SGD: {e_s} of {epochs} epochs x{epochs / e_s:g} (num_threads={cores})"}


def run_reference(args, rank: int) -> dict | None:
    if rank != 0:
        return None
    n, dim, _, _, _, k, epochs = CONFIGS[args.config]
    vals = []
    cb = None
    # the host-core reference needs no warm-up: every step is a fresh bounded sample
    for _ in range(max(args.steps, 1)):
        cb = cpu_sample(args.config)
        vals.append(cb["value"])
    v = float(np.median(vals))
    cb["value"] = v
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Gaussian mixture)",
            "config": {"workload": f"{args.config}: n={n} dim={dim} k={k} out_dim=2 epochs={epochs}"},
            "cpu_baseline": cb, "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def trustworthiness_dev(X: np.ndarray, Y: np.ndarray, k: int, queries: np.ndarray, batch: int = 8) -> float:
    """Trustworthiness(k) of layout Y for data X over the query rows (FP64
    squared distances, ranks with ties broken by index, the whole data set as
    candidates), computed with torch on the GPU: a layout-quality measure."""
    import torch

    n = X.shape[0]
    Xd = torch.as_tensor(np.ascontiguousarray(X), device="cuda").to(torch.float64)
    Yd = torch.as_tensor(np.ascontiguousarray(Y), device="cuda").to(torch.float64)
    ar = torch.arange(n, device="cuda")
    total = 0.0
    for s in range(0, len(queries), batch):
        qi = torch.as_tensor(queries[s:s + batch], device="cuda", dtype=torch.long)
        rows = torch.arange(len(qi), device="cuda")
        dX = ((Xd[None, :, :] - Xd[qi][:, None, :]) ** 2).sum(-1)
        dY = ((Yd[None, :, :] - Yd[qi][:, None, :]) ** 2).sum(-1)
        dY[rows, qi] = float("inf")
        cand = torch.sort(torch.topk(dY, min(k + 8, n - 1), dim=1, largest=False).indices, dim=1).values
        nb = torch.gather(cand, 1, torch.argsort(torch.gather(dY, 1, cand), dim=1, stable=True))[:, :k]
        dj = torch.gather(dX, 1, nb)
        for t in range(k):
            closer = (dX < dj[:, t:t + 1]) | ((dX == dj[:, t:t + 1]) & (ar[None, :] < nb[:, t:t + 1]))
            closer[rows, qi] = False
            total += float(torch.clamp(closer.sum(1) + 1 - k, min=0).sum())
    return 1.0 - 2.0 / (len(queries) * k * (2.0 * n - 3.0 * k - 1.0)) * total


def precision_study(cfg: str) -> dict:
    """Per-stage error of the FP32 path against the FP64 device path on the
    benchmark workload (same data, rounded once to float32):
    - kNN: the 3xFP16 (default) and 3xTF32 tensor-core searches on float32
      data against the FP64 search of the same points: rows and entries with
      the same neighbour indices, largest relative distance error;
    - similarities, union, schedule: float32 and float64 runs of each stage on
      the same FP64 neighbour lists: largest relative weight difference, edge
      counts, largest relative epochs_per_sample difference;
    - layout: the full float32 pipeline (FP32 2-d SGD kernel) and the full
      float64 pipeline (FP64 generic kernel), each scored by the fuzzy
      cross-entropy over the FP64 union graph (device loss, with its constant)
      and trustworthiness (k = 15, 10,000 seeded queries)."""
    import umappp_b200 as U

    n, dim, _, _, _, k, epochs = CONFIGS[cfg]
    X32 = make_data(cfg)
    X64 = X32.astype(np.float64)
    out = {"workload": cfg}
    t0 = time.time()
    idx64, d64 = U.knn(X64, k)
    out["knn_fp64_s"] = round(time.time() - t0, 2)
    knn = {}
    for kind, env in (("fp16x3", None), ("tf32x3", "tf32")):
        if env:
            os.environ["UMAPB_KNN_TC_KIND"] = env
        try:
            t0 = time.time()
            idx, d = U.knn(X32, k)
            secs = time.time() - t0
        finally:
            os.environ.pop("UMAPB_KNN_TC_KIND", None)
        rel = np.abs(d.astype(np.float64) - d64) / np.maximum(d64, 1e-300)
        knn[kind] = {"rows_equal": round(float(np.mean(np.all(idx == idx64, axis=1))), 6),
                     "entries_equal": round(float(np.mean(idx == idx64)), 7),
                     "max_rel_distance_error": float(rel[idx == idx64].max()), "seconds": round(secs, 2)}
    out["knn"] = knn
    nl32 = (idx64, d64.astype(np.float32))
    p, i, w32 = U.neighbor_similarities(nl32)
    _, _, w64 = U.neighbor_similarities((idx64, d64))
    out["similarities_max_rel_error"] = float(np.max(np.abs(w32 - w64) / np.maximum(w64, 1e-300)))
    g32 = U.combine_neighbor_sets((p, i, w32))
    g64 = U.combine_neighbor_sets((p, i, w64))
    e32 = U.similarities_to_epochs(g32, epochs, 5.0)
    e64 = U.similarities_to_epochs(g64, epochs, 5.0)
    same = (len(e32.edge_targets) == len(e64.edge_targets) and np.array_equal(e32.edge_targets, e64.edge_targets))
    out["union_edges"] = {"fp32": int(len(g32[1])), "fp64": int(len(g64[1]))}
    out["schedule"] = {"edges_fp32": int(len(e32.edge_targets)), "edges_fp64": int(len(e64.edge_targets)),
                       "same_edges": bool(same)}
    if same:
        out["schedule"]["max_rel_epochs_per_sample_error"] = float(np.max(
            np.abs(e32.epochs_per_sample.astype(np.float64) - e64.epochs_per_sample) / e64.epochs_per_sample))
    a, b = U.find_ab(1.0, 0.1)
    queries = np.sort(np.random.default_rng(123).choice(n, size=min(10000, n), replace=False))
    layout = {}
    for name, X, dt in (("fp32", X32, np.float32), ("fp64", X64, np.float64)):
        Y = np.zeros((n, 2), dt)
        st = U.initialize_from_data(X, 2, Y, U.Options(num_neighbors=k, num_epochs=epochs))
        st.run(Y)
        ms = st.stage_ms()
        ce = U.loss_grad(g64, Y.astype(np.float64), a, b, with_constant=True)[0]
        layout[name] = {"cross_entropy": ce, "trustworthiness": round(trustworthiness_dev(X64, Y, 15, queries), 6),
                        "sgd_ms": round(ms["sgd"], 1), "knn_ms": round(ms["knn"], 1)}
    layout["fp32_vs_fp64_cross_entropy"] = round(
        (layout["fp32"]["cross_entropy"] - layout["fp64"]["cross_entropy"]) / layout["fp64"]["cross_entropy"], 6)
    out["layout"] = layout
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="mixture_1m", choices=sorted(CONFIGS) + ["batch64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batch64 sub-object of the default line")
    ap.add_argument("--precision-study", action="store_true",
                    help="print the per-stage FP32-vs-FP64 comparison on the workload and exit")
    ap.add_argument("--no-precision", action="store_true", help="skip the precision sub-object of the default line")
    args = ap.parse_args()
    if args.precision_study:
        print(json.dumps({"precision_study": precision_study(args.config)}), flush=True)
        return

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    if args.impl == "reference":
        if args.config == "batch64":
            if rank == 0:
                print(json.dumps({"impl": "reference", "unavailable": "batch64 is a device-only mode without a "
                                  "reference counterpart"}), flush=True)
            return
        out = run_reference(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        return

    import torch
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        out = run_batch(args, rank, world) if args.config == "batch64" else run_ours(args, rank, world)
        if world == 1 and args.config == "mixture_1m" and not args.no_batch and out is not None:
            # the batched mode (64 independent instances in one call) beside the headline
            b = run_batch(argparse.Namespace(steps=2, warmup=1), rank, world)
            out["batch64"] = {k_: b[k_] for k_ in ("value", "unit", "sequential_plain_s", "speedup_vs_sequential",
                                                   "gpu_launches", "sequential_gpu_launches")}
            out["batch64"]["workload"] = b["config"]["workload"]
        if world == 1 and args.config == "mixture_1m" and not args.no_precision and out is not None:
            # per-stage error of the FP32 path against the FP64 device path (after the timed region)
            out["precision"] = precision_study(args.config)
        if rank == 0 and out is not None:
            if world == 1 and not args.no_cpu_baseline and args.config != "batch64":
                out["cpu_baseline"] = cpu_sample(args.config)
            print(json.dumps(out), flush=True)
    finally:
        if world > 1:
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
