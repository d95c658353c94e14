"""Benchmark of the exact painter: receiver-source paths per second on one B200.

Workload (default `terrain`): the 16 km^2 terrain square at full size (2048 x 2048 receivers at
1.953 m, fBm DEM at 5 m posts with +-40 m relief, Voronoi ground factor over 200 cells, 20,000 road
and rail segments split into ~4.0 M one-metre point sources, 30,000 polygon buildings, favourable
probability 0.5 per sector). Painting the whole square is ~10^13 paths, so a step paints one
seeded 16 x 8 receiver tile of the grid against one eighth of the source list (~0.5 M sources,
~64 M paths); eight consecutive steps paint a tile against every source. Workload `road` paints
the whole 1 km road square (128 x 128 receivers x 77,354 point sources) per step. Workload
`flights` paints the Doc 29 aircraft grid (1024^2 cells x 10^5 flight segments) with loudness.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload ...]

`value` is paths per second of device time (CUDA events around the painting kernels, inputs
resident); `e2e` is the same metric through the C ABI call with host buffers (receiver set-up,
host-device copies and the read-back of the cell levels and histogram inside the timed region).
L2 is flushed between steps (a 256 MB write). `roofline` rates the main painting kernel: the
kernel is compute-bound, so its work is counted in FP32 operations from the per-path work counters
the kernel returns (an operation model, below) against the nominal FP32 peak; `roofline_hbm`
gives its algorithmic bytes against the measured HBM bandwidth with the DRAM traffic ncu saw.

`--impl reference` times the reference's CPU path on the host cores instead: the reference is Rust
and cannot be built on this image, so its FP64 restatement (oracle/) stands in for it, on all
host threads, on a bounded sample of the same workload.
Under torchrun each rank paints its own receiver sample (replicas; the path shards by receiver
tiles with no exchange) and rank 0 prints the JSON line with the max time over ranks.
"""

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "receiver–source paths/s at ≤0.1 dB vs FP64 oracle; surrogate vs exact, 1 B200"
SM_COUNT, FP32_LANES, MUFU_LANES = 148, 128, 16
NOMINAL_SM_MHZ = 1965.0

# Operation model of one path (FP32 operations; SFU operations apart), from the exact path code:
#   a segment-edge test 12, a profile vertex (terrain lattice step or roof vertex: position,
#   height, segment moments, ground share) 20, a crossing (chainage, height, roof pairing) 10, a
#   diffraction candidate (hull test and push) 12, and per path the ground attenuation of two
#   states x 8 bands x 40, air absorption 8, geometry 30 and the three period sums 3 x 8 x 4.
#   Diffraction's own arithmetic (path differences in FP64, ~500 operations per diffracted
#   state) is not counted, so the model is a lower bound of the work.
OPS = dict(edge_test=12, vertex=20, crossing=10, candidate=12, path=2 * 8 * 40 + 8 + 30 + 3 * 8 * 4)
# SFU operations per path: 5 per band and state (exp, sqrt, log10 of the ground term), 8 exp of
# air absorption, 3 x 8 exp of the period energies.
SFU_PER_PATH = 2 * 8 * 5 + 8 + 3 * 8


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="terrain", choices=["terrain", "road", "flights", "surrogate", "surrogate_terrain", "tiles", "loudness",
                             "flight_sums", "horizons"])
    ap.add_argument("--tiles", type=int, default=32, help="tiles workload: tiles per batch, drawn from the 4096")
    ap.add_argument("--flights", type=int, default=2000, help="flights workload: flights (a small case for profiling)")
    ap.add_argument("--cells-side", type=int, default=1024, help="flights workload: receivers per side")
    ap.add_argument("--lattice-side", type=int, default=64,
                    help="flight_sums workload: lattice points per side of the square")
    ap.add_argument("--slices", type=int, default=8, help="terrain: source-list slices (a step paints one)")
    ap.add_argument("--sources", type=int, default=0,
                    help="paint only the first N sources (a small case for profiling; 0: all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true",
                    help="terrain: leave out the surrogate leg (its training launches many kernels)")
    ap.add_argument("--oracle-cells", type=int, default=32,
                    help="terrain: cells of the timed steps checked against the FP64 oracle")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def combine_ranks(timing, paths, device):
    """Replicas: every rank's times become the max over ranks (device times and wall time), the
    path counts their sum. Returns the total paths; `timing` is updated in place."""
    import torch
    import torch.distributed as tdist
    t = torch.tensor([timing["kernel_ms"], timing["wall_s"], timing["paint_ms"]], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    timing["kernel_ms"], timing["wall_s"], timing["paint_ms"] = float(t[0]), float(t[1]), float(t[2])
    tp = torch.tensor([float(paths)], dtype=torch.float64, device=device)
    tdist.all_reduce(tp)
    return int(tp[0])


def workload(name, rank, slices, sources):
    """The scene and a list of steps (each a list of grids painted in that step)."""
    from quietmap_b200 import scenes
    if name == "road":
        scene, full = scenes.road_square()
        n_src = min(sources, len(scene.sources)) if sources else len(scene.sources)
        full.source_begin, full.source_end = 0, n_src
        desc = dict(workload=f"road square 1 km: 128x128 receivers at 7.8125 m x {n_src} point sources from 400 "
                             "road segments, 300 buildings, flat G=0.5, homogeneous, one whole grid per step")
        return scene, [[full]], desc
    scene, full = scenes.terrain_square()
    n_all = len(scene.sources)
    n_src = min(sources, n_all) if sources else n_all
    slices = max(1, slices)
    per = (n_src + slices - 1) // slices
    steps = [[g] for g in scenes.terrain_tile_steps(full, n_src, seed=1000 + rank, slices=slices)]
    desc = dict(workload=f"terrain square 16 km^2 (2048^2 grid at 1.953 m, fBm DEM, 30,000 buildings, "
                         f"{n_all} point sources from 20,000 road/rail segments, p=0.5): a step is one seeded "
                         f"16x8 receiver tile x one 1/{slices} slice ({per} sources) of the source list",
                scene_sources=n_all)
    return scene, steps, desc


class ClockSampler:
    """nvidia-smi clocks sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._thread = None

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([v.strip() for v in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def measured_peaks():
    """The pool's measured peaks (driver-written), else the earlier measurement on this pool
    (6.65 TB/s copy, 1.59 PFLOP/s bf16), marked as the fallback."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return dict(json.load(f), source="measured")
    except (OSError, ValueError):
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "source": "fallback"}


# DRAM bytes per path of the painting kernel, from one ncu capture of the current kernel on a small
# case of the workload (one 16 x 8 tile x the first 20,000 sources, 2.56 M paths:
# dram__bytes_read.sum 19.88 GB + dram__bytes_write.sum 27.09 GB), scaled by paths to a full
# launch. None where no capture of the current kernel exists.
DRAM_BYTES_PER_PATH = {"terrain": 18347.0, "road": None}


def stratified_sources(grid, m, seed):
    """`m` source indices spread evenly over the grid's source range from a seeded offset: every
    part of the slice is sampled, near and far sources alike."""
    n = grid.source_end - grid.source_begin
    u = np.random.default_rng(seed).uniform()
    return grid.source_begin + np.minimum(((np.arange(m) + u) * (n / m)).astype(np.int64), n - 1)


def cpu_sample(scene, g, seconds, seed=17):
    """The oracle's bounded sample of a timed step: the step's receivers (its whole tile) against a
    stratified, seeded subsample of the step's source slice, grown until the oracle takes about
    `seconds` on all host threads. Returns (oracle scene, grid, sources sampled, threads)."""
    from dataclasses import replace
    from oracle import oracle
    threads = oracle.threads()
    n_slice = g.source_end - g.source_begin

    def sub(m):
        idx = stratified_sources(g, m, seed)
        return oracle.OracleScene(replace(scene, sources=scene.sources[idx])), replace(g, source_begin=0,
                                                                                     source_end=len(idx)), idx
    m = 64
    while True:
        ora, grid, _ = sub(m)
        t0 = time.perf_counter()
        ora.paint_grid(grid, nthreads=threads)
        dt = time.perf_counter() - t0
        if dt > seconds / 4 or m >= n_slice:
            break
        m = min(int(m * max(2.0, seconds / 4 / max(dt, 1e-3))), n_slice)
    m = min(n_slice, max(1, int(m * seconds / max(dt, 1e-3))))
    ora, grid, idx = sub(m)
    return ora, grid, idx, threads


def cpu_run(ora, grid, threads):
    t0 = time.perf_counter()
    ora.paint_grid(grid, nthreads=threads)
    return time.perf_counter() - t0


def cpu_work(ora, scene, grid, idx, n_pairs=256, seed=19):
    """The oracle's work per path on a seeded subset of the sample's pairs: crossings, profile
    vertices and diffraction candidates (qmo_path_counts)."""
    rng = np.random.default_rng(seed)
    cells = rng.integers(0, grid.cells, n_pairs)
    srcs = rng.integers(0, len(idx), n_pairs)
    rxy = grid.receiver_xy()[cells]
    sxy = np.stack([scene.sources["x"][idx[srcs]], scene.sources["y"][idx[srcs]]], axis=1)
    counts = ora.path_counts(sxy, rxy)
    return {"crossings": float(counts[:, 0].mean()), "vertices": float(counts[:, 1].mean()),
            "candidates": float(counts[:, 2].mean()), "pairs_counted": n_pairs}


def cpu_description(grid, g, idx, dt):
    return (f"the first timed step's {grid.cells} receivers x {len(idx)} of its {g.source_end - g.source_begin} "
            f"sources (stratified, seeded) = {grid.cells * len(idx)} paths, {dt:.1f} s")


def cpu_baseline(scene, g, seconds=12.0):
    """The FP64 oracle on all host threads: paths/s on a bounded sample of a timed step."""
    ora, grid, idx, threads = cpu_sample(scene, g, seconds)
    dt = cpu_run(ora, grid, threads)
    return dict(value=grid.cells * len(idx) / dt, unit="paths/s", cores=threads, kind="port",
                sample=cpu_description(grid, g, idx, dt), per_path=cpu_work(ora, scene, grid, idx))


def algorithmic_bytes(scene, grid, n_src):
    """Bytes one painting launch must move at least: its source slice (128 B a record), the
    outlines and vertices, the DEM (altitude and ground factor, 4 B each), and the partial sums it
    writes (9 floats per cell and source chunk are bounded by the cell outputs: 36 B a cell)."""
    b = n_src * 128 + scene.outlines.nbytes + scene.vertices.nbytes
    if scene.dem_altitude is not None:
        b += scene.dem_altitude.size * 8
    return b + grid.nx * grid.ny * 36


def main():
    args = parse()
    rank, world, local = dist_env()
    if world > 1:
        import torch
        import torch.distributed as tdist
        from datetime import timedelta
        backend = "nccl" if args.impl == "ours" else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        tdist.init_process_group(backend, timeout=timedelta(seconds=600))
    if args.impl == "reference":
        return reference_arm(args, rank, world)
    if args.workload == "flights":
        return flights(args, rank, world, local)
    if args.workload == "surrogate":
        return surrogate(args, rank, world, local)
    if args.workload == "surrogate_terrain":
        return surrogate_terrain(args, rank, world, local)
    if args.workload == "tiles":
        return tile_batch(args, rank, world, local)
    if args.workload == "loudness":
        return loudness(args, rank, world, local)
    if args.workload == "flight_sums":
        return flight_sums(args, rank, world, local)
    if args.workload == "horizons":
        return horizons(args, rank, world, local)
    import torch
    from quietmap_b200 import native
    scene, steps, desc = workload(args.workload, rank, args.slices, args.sources)
    ctx = native.Context(local if world > 1 else 0)
    dev = ctx.scene(scene)
    torch.cuda.set_device(local if world > 1 else 0)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2

    work = dict(paths=0, edge_tests=0, vertices=0, candidates=0, crossings=0, failed_paths=0)
    timing = dict(kernel_ms=0.0, paint_ms=0.0, wall_s=0.0, launches=0, paint_launches=0, alg_bytes=0, paths_timed=0)
    timed_dba = {}  # step index -> the exact painter's cell dBA (the surrogate leg compares with it)

    def step(i):
        for g in steps[i % len(steps)]:
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, dba, _, _, st = dev.paint_grid(g)
            timed_dba[i] = dba
            timing["wall_s"] += time.perf_counter() - t0
            timing["kernel_ms"] += st["kernel_ms"]
            timing["paint_ms"] += st["paint_ms"]
            timing["launches"] += 2 + (2 if st["failed_paths"] else 0)
            timing["paint_launches"] += 1
            timing["alg_bytes"] += algorithmic_bytes(scene, g, g.source_end - g.source_begin)
            timing["paths_timed"] += st["paths"]
            for k in work:
                work[k] += st[k]

    for i in range(args.warmup):
        step(i)
    for d in (work, timing):
        for k in d:
            d[k] = 0
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            step(args.warmup + i)
        torch.cuda.synchronize()
    if world > 1:
        total_paths = combine_ranks(timing, work["paths"], "cuda")
    else:
        total_paths = work["paths"]
    if rank == 0:
        clk = clocks.summary()
        peaks = measured_peaks()
        cells_per_call = steps[0][0].cells
        calls = sum(len(steps[(args.warmup + i) % len(steps)]) for i in range(args.steps))
        paths = max(work["paths"], 1)
        ops = (OPS["edge_test"] * work["edge_tests"] + OPS["vertex"] * work["vertices"]
               + OPS["crossing"] * work["crossings"] + OPS["candidate"] * work["candidates"]
               + OPS["path"] * work["paths"])
        paint_s = timing["paint_ms"] / 1e3
        fp32_peak = SM_COUNT * FP32_LANES * 2 * NOMINAL_SM_MHZ * 1e6 / 1e12
        achieved = ops / paint_s / 1e12 if paint_s > 0 else None
        sfu_peak = SM_COUNT * MUFU_LANES * NOMINAL_SM_MHZ * 1e6
        caps = "terrain" if args.workload == "terrain" else "road"
        traffic_per_path = DRAM_BYTES_PER_PATH.get(caps)
        hbm_peak = peaks.get("hbm_gbs")
        alg_gbs = timing["alg_bytes"] / paint_s / 1e9 if paint_s > 0 else None
        line = {
            "metric": METRIC,
            "value": total_paths / (timing["kernel_ms"] / 1e3),
            "unit": "paths/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": timing["kernel_ms"] / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (f64 for path differences and crossing chainage)",
            "data": "synthetic (seeded generator of the workload's geometry)",
            "config": dict(desc, paths_per_step=work["paths"] // max(args.steps, 1),
                           parallelism=f"replicas x{world}", l2="flushed between steps (256 MB write)"),
            "e2e": {"value": total_paths / timing["wall_s"], "unit": "paths/s",
                    "h2d_bytes_per_step": calls * cells_per_call * 8 // args.steps,
                    "d2h_bytes_per_step": calls * (cells_per_call * 40 + 1800 * 4) // args.steps},
            "gpu_launches": timing["launches"],
            "clocks": clk,
            "roofline": {
                "kernel": f"paint_grid_kernel<Caps{caps.capitalize()}>",
                "bound": "fp32",
                "achieved": achieved,
                "peak": fp32_peak,
                "unit": "TFLOP/s",
                "frac": achieved / fp32_peak if achieved else None,
                "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1965 MHz); the measured peaks file "
                               "holds no FP32 figure",
                "ops_per_path": ops / paths,
                "sfu_frac": (SFU_PER_PATH * work["paths"] / paint_s / sfu_peak) if paint_s > 0 else None,
                "traffic": traffic_per_path * work["paths"] / max(timing["paint_launches"], 1)
                if traffic_per_path else None,
                "launch_ms": timing["paint_ms"] / max(timing["paint_launches"], 1),
            },
            "roofline_hbm": {
                "bound": "hbm",
                "achieved": alg_gbs,
                "peak": hbm_peak,
                "unit": "GB/s",
                "frac": alg_gbs / hbm_peak if (alg_gbs and hbm_peak) else None,
                "peak_source": peaks.get("source"),
                "algorithmic_bytes_per_launch": timing["alg_bytes"] / max(timing["paint_launches"], 1),
                "traffic": traffic_per_path * work["paths"] / max(timing["paint_launches"], 1)
                if traffic_per_path else None,
            },
            "per_path": {k: work[k] / paths for k in ("crossings", "edge_tests", "vertices", "candidates")},
            "failed_paths_rerun": work["failed_paths"],
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(scene, steps[args.warmup % len(steps)][0])
    if args.workload == "terrain" and not args.no_surrogate and world == 1:
        sur = surrogate_leg(args, ctx, dev, scene, steps, timed_dba, timing, flush, rank)
        if rank == 0:
            line["surrogate"] = sur
    if rank == 0:
        print(json.dumps(line), flush=True)
    dev.close()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def oracle_cells(scene, jobs, threads):
    """The FP64 oracle's dBA of each (grid, cell) job, one host thread a cell (the oracle's calls
    release the GIL), all threads busy."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle
    ora = oracle.OracleScene(scene)

    def one(job):
        g, c = job
        e, _, _ = ora.paint_grid(g, c, c + 1, nthreads=1)
        return 10.0 * np.log10(e[0].sum())
    with ThreadPoolExecutor(max_workers=threads) as pool:
        return np.array(list(pool.map(one, jobs)))


def surrogate_leg(args, ctx, dev, scene, steps, exact_dba, timing, flush, rank):
    """The learned surrogate on the same timed steps as the exact painter. The network is trained
    first (untimed): exact paths of 12 coarse receiver grids x 25,000-source slices (80 M rows, two
    per path), paths shorter than 200 m left to the exact path. Its painting is timed on the same
    steps (L2 flushed before each); its speed-up is against the exact painter's time on those
    steps. Seeded cells of the timed steps are checked against the FP64 oracle, for the surrogate
    and for the exact painter alike."""
    import torch
    from oracle import oracle
    from quietmap_b200 import native, scenes
    ns = len(scene.sources)
    spacing = steps[0][0].spacing
    cells = steps[0][0].cells
    grids = [scenes.Grid(origin=(spacing // 2 + 131 * k, spacing // 2 + 257 * k), spacing=spacing * 128, nx=16, ny=16,
                         source_begin=(k * 331_001) % (ns - 25_000), source_end=(k * 331_001) % (ns - 25_000) + 25_000)
             for k in range(12)]
    net = native.Surrogate(ctx, seed=1)
    exact_within_m = 200.0
    t0 = time.perf_counter()
    hist, n_train = net.train(dev, grids, epochs=6, batch=16384, learning_rate=2e-3, seed=3, max_samples=80_000_000,
                              exact_within_m=exact_within_m)
    train_s = time.perf_counter() - t0
    for i in range(args.warmup):
        dev.paint_grid_surrogate(steps[i % len(steps)][0], net)
    s_ms = 0.0
    paths = taken = 0
    sur_dba = {}
    torch.cuda.synchronize()
    with ClockSampler(0) as clocks:
        for i in range(args.steps):
            g = steps[(args.warmup + i) % len(steps)][0]
            flush.zero_()
            torch.cuda.synchronize()
            _, dba, _, _, st = dev.paint_grid_surrogate(g, net)
            s_ms += st["kernel_ms"]
            paths += st["paths"]
            taken += st["surrogate_paths"]
            sur_dba[args.warmup + i] = dba
    net.close()
    # Against the exact painter on every timed cell.
    vs_exact = np.concatenate([np.abs(sur_dba[k] - exact_dba[k]) for k in sur_dba])
    # Against the FP64 oracle on seeded cells of the timed steps.
    rng = np.random.default_rng(23)
    keys = sorted(sur_dba)
    jobs, picks = [], []
    for j in range(args.oracle_cells):
        k = keys[j % len(keys)]
        c = int(rng.integers(0, cells))
        jobs.append((steps[k % len(steps)][0], c))
        picks.append((k, c))
    t0 = time.perf_counter()
    ref = oracle_cells(scene, jobs, oracle.threads())
    oracle_s = time.perf_counter() - t0
    sur_err = np.abs(np.array([sur_dba[k][c] for k, c in picks]) - ref)
    exa_err = np.abs(np.array([exact_dba[k][c] for k, c in picks]) - ref)
    exact_paths_per_s = timing["paths_timed"] / (timing["kernel_ms"] / 1e3)
    value = paths / (s_ms / 1e3)

    def stats(e):
        return {"p50": float(np.percentile(e, 50)), "p99": float(np.percentile(e, 99)), "max": float(e.max())}
    return {
        "value": value, "unit": "paths/s", "exact_value": exact_paths_per_s, "speedup_vs_exact": value / exact_paths_per_s,
        "ms_per_step": s_ms / args.steps, "surrogate_share": taken / max(paths, 1),
        "dtype": "bf16 network (fp32 accumulate, tcgen05), f32 path code",
        "cell_dba_error_vs_oracle_db": dict(stats(sur_err), cells=len(sur_err)),
        "exact_cell_dba_error_vs_oracle_db": dict(stats(exa_err), cells=len(exa_err)),
        "cell_dba_error_vs_exact_db": dict(stats(vs_exact), cells=int(vs_exact.size)),
        "oracle_seconds": oracle_s,
        "training": {"samples": int(n_train), "epochs": 6, "seconds": train_s, "loss": [float(v) for v in hist],
                     "exact_within_m": exact_within_m},
        "clocks": clocks.summary(),
    }


# Doc 29 operation model per (cell, segment) pair in reach: about 150 FP32 operations and 10 SFU
# operations (closest point, NPD interpolation in log distance, power-row lerp, speed, finite
# segment, lateral and installation corrections, the energy and its compensated sum).
DOC29_OPS_PER_PAIR, DOC29_SFU_PER_PAIR = 150, 10
ZWICKER_BYTES_PER_CELL = 28 * 4 + 4


def flights(args, rank, world, local):
    """Doc 29 flights (1024^2 cells at 100 m x 2000 flights x 50 segments) with loudness."""
    import torch
    from quietmap_b200 import native, scenes
    f = scenes.flights_square(seed=3 + rank, n_flights=args.flights, receivers=args.cells_side)
    ctx = native.Context(local if world > 1 else 0)
    cells = f.grid["nx"] * f.grid["ny"]
    for _ in range(args.warmup):
        ctx.flight_grid(f)
    torch.cuda.synchronize()
    k_ms = z_ms = 0.0
    in_reach = 0
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _, _, _, st = ctx.flight_grid(f, stats=True)
            k_ms += st["kernel_ms"]
            z_ms += st["loudness_ms"]
            in_reach += st["pairs_in_reach"]
        wall = time.perf_counter() - t0
    if rank == 0:
        peaks = measured_peaks()
        device_s = (k_ms + z_ms) / 1e3
        fp32_peak = SM_COUNT * FP32_LANES * 2 * NOMINAL_SM_MHZ * 1e6 / 1e12
        achieved = DOC29_OPS_PER_PAIR * in_reach / (k_ms / 1e3) / 1e12
        line = {
            "metric": "Doc 29 cells/s (cell x flight-segment pairs with Zwicker loudness), 1 B200",
            "value": cells * args.steps / device_s, "unit": "cells/s",
            "pairs_in_reach_per_s": in_reach / (k_ms / 1e3),
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (k_ms + z_ms) / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded flights and NPD tables)",
            "config": {"workload": f"{args.cells_side}^2 cells at 100 m x {args.flights} flights x 50 segments, 10 types, "
                                   "reach 25 km",
                       "pairs_in_reach_per_step": in_reach // args.steps},
            "e2e": {"value": cells * args.steps / wall, "unit": "cells/s",
                    "h2d_bytes_per_step": len(f.segments) * 48 + len(f.types) * f.types.itemsize,
                    "d2h_bytes_per_step": cells * (4 + 28 * 4 + 4)},
            "roofline": {"kernel": "flight_grid_kernel", "bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                         "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                         "peak_source": "nominal FP32 (148 SMs x 128 lanes x 2 x 1965 MHz)",
                         "ops_per_pair": DOC29_OPS_PER_PAIR, "launch_ms": k_ms / args.steps},
            "roofline_loudness": {"kernel": "zwicker_kernel", "bound": "hbm",
                                  "achieved": ZWICKER_BYTES_PER_CELL * cells * args.steps / (z_ms / 1e3) / 1e9,
                                  "peak": peaks.get("hbm_gbs"), "unit": "GB/s", "launch_ms": z_ms / args.steps,
                                  "peak_source": peaks.get("source")},
            "clocks": clocks.summary(), "gpu_launches": 2 * args.steps,
        }
        if line["roofline_loudness"]["peak"]:
            line["roofline_loudness"]["frac"] = line["roofline_loudness"]["achieved"] / line["roofline_loudness"]["peak"]
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle
            n = 64
            t0 = time.perf_counter()
            oracle.flight_grid(f, 0, n)
            dt = time.perf_counter() - t0
            n = max(n, min(cells, int(n * 12.0 / max(dt, 1e-3))))
            t0 = time.perf_counter()
            oracle.flight_grid(f, 0, n)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = dict(value=n / dt, unit="cells/s", cores=oracle.threads(), kind="port",
                                        sample=f"the first {n} cells against every segment ({dt:.1f} s)")
        print(json.dumps(line), flush=True)
    ctx.close()


def surrogate(args, rank, world, local):
    """The surrogate painter against the exact painter on the config-1 style 2048^2 square (the
    1 km road square with 2048 x 2048 receivers at 0.469 m): the network is trained first (50 M
    exact paths of the same geometry, untimed), then each step paints one seeded 16 x 8 tile
    against every source with both painters."""
    import torch
    from quietmap_b200 import native, scenes
    scene, full = scenes.road_square(receivers=2048)
    ctx = native.Context(local if world > 1 else 0)
    dev = ctx.scene(scene)
    net = native.Surrogate(ctx, seed=1)

    def coarse(n, off):
        sp = (scene.extent_steps[0] - 2 * off) // n
        return scenes.Grid(origin=(off, off), spacing=sp, nx=n, ny=n)

    t0 = time.perf_counter()
    hist, n_train = net.train(dev, [coarse(24, 37 + 101 * k) for k in range(4)], epochs=3, batch=16384,
                              learning_rate=2e-3, seed=3, max_samples=50_000_000)
    train_s = time.perf_counter() - t0
    # Held-out paths: the network against the exact labels.
    f, lab, ok = dev.surrogate_samples(scenes.Grid(origin=(555, 777), spacing=7001, nx=4, ny=4, source_end=40000))
    err = np.abs(net.forward(f[ok]) - lab[ok])
    rng = np.random.default_rng(2000 + rank)
    tiles = []
    for _ in range(max(args.steps + args.warmup, 1)):
        tx, ty = int(rng.integers(0, full.nx // 16)), int(rng.integers(0, full.ny // 8))
        tiles.append(scenes.Grid(origin=(full.origin[0] + tx * 16 * full.spacing, full.origin[1] + ty * 8 * full.spacing),
                                 spacing=full.spacing, nx=16, ny=8))
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    for i in range(args.warmup):
        dev.paint_grid_surrogate(tiles[i], net)
        dev.paint_grid(tiles[i])
    s_ms = e_ms = 0.0
    paths = taken = 0
    cell_err = []
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            g = tiles[args.warmup + i]
            flush.zero_()
            torch.cuda.synchronize()
            sb, sdba, _, _, sst = dev.paint_grid_surrogate(g, net)
            flush.zero_()
            torch.cuda.synchronize()
            eb, edba, _, _, est = dev.paint_grid(g)
            s_ms += sst["kernel_ms"]
            e_ms += est["kernel_ms"]
            paths += sst["paths"]
            taken += sst["surrogate_paths"]
            cell_err.append(np.abs(sdba - edba))
    cell_err = np.concatenate(cell_err)
    if rank == 0:
        value, exact = paths / (s_ms / 1e3), paths / (e_ms / 1e3)
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": s_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network (fp32 accumulate), f32 path code",
            "data": "synthetic (seeded road square geometry)",
            "config": {"workload": "surrogate painter, road square 1 km with 2048^2 receivers (0.469 m): a step is one "
                                   "seeded 16x8 tile x 77,354 point sources", "l2": "flushed between painters"},
            "exact_value": exact, "speedup_vs_exact": value / exact, "surrogate_share": taken / max(paths, 1),
            "path_error_db": {"p50": float(np.percentile(err, 50)), "p99": float(np.percentile(err, 99)),
                              "samples": int(err.size)},
            "cell_dba_error_db": {"p50": float(np.median(cell_err)), "p99": float(np.percentile(cell_err, 99)),
                                  "max": float(cell_err.max())},
            "training": {"samples": int(n_train), "epochs": 3, "seconds": train_s, "loss": [float(v) for v in hist]},
            "clocks": clocks.summary(), "gpu_launches": args.steps * 5,
        }), flush=True)
    ctx.close()


def surrogate_terrain(args, rank, world, local):
    """The surrogate painter against the exact painter on the terrain square (full size: fBm DEM,
    30,000 buildings, 3.99 M point sources, favourable p = 0.5): the network is trained first
    (untimed) on exact paths of 12 coarse receiver grids x 25,000-source slices (80 M rows, two
    per path), leaving paths shorter than 200 m to the exact path, then each step paints one
    seeded 16 x 8 tile against one 1/8 slice of the sources with both painters."""
    import torch
    from quietmap_b200 import native, scenes
    scene, full = scenes.terrain_square()
    ctx = native.Context(local if world > 1 else 0)
    dev = ctx.scene(scene)
    net = native.Surrogate(ctx, seed=1)
    ns = len(scene.sources)
    grids = [scenes.Grid(origin=(full.origin[0] + 131 * k, full.origin[1] + 257 * k), spacing=full.spacing * 128,
                         nx=16, ny=16, source_begin=(k * 331_001) % (ns - 25_000),
                         source_end=(k * 331_001) % (ns - 25_000) + 25_000) for k in range(12)]
    t0 = time.perf_counter()
    exact_within_m = 200.0
    hist, n_train = net.train(dev, grids, epochs=6, batch=16384, learning_rate=2e-3, seed=3, max_samples=80_000_000,
                              exact_within_m=exact_within_m)
    train_s = time.perf_counter() - t0
    f, lab, ok = dev.surrogate_samples(scenes.Grid(origin=(full.origin[0] + 555, full.origin[1] + 777),
                                                   spacing=full.spacing * 300, nx=4, ny=4, source_begin=0,
                                                   source_end=20000))
    err = np.abs(net.forward(f[ok]) - lab[ok])
    _, steps, _ = workload("terrain", rank, args.slices, 0)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    for i in range(args.warmup):
        dev.paint_grid_surrogate(steps[i][0], net)
    s_ms = e_ms = 0.0
    paths = taken = 0
    cell_err = []
    with ClockSampler(local) as clocks:
        for i in range(args.steps):
            g = steps[args.warmup + i][0]
            flush.zero_()
            torch.cuda.synchronize()
            _, sdba, _, _, sst = dev.paint_grid_surrogate(g, net)
            flush.zero_()
            torch.cuda.synchronize()
            _, edba, _, _, est = dev.paint_grid(g)
            s_ms += sst["kernel_ms"]
            e_ms += est["kernel_ms"]
            paths += sst["paths"]
            taken += sst["surrogate_paths"]
            cell_err.append(sdba - edba)
    cell_signed = np.concatenate(cell_err)
    cell_err = np.abs(cell_signed)
    if rank == 0:
        value, exact = paths / (s_ms / 1e3), paths / (e_ms / 1e3)
        print(json.dumps({
            "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": s_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "bf16 network (fp32 accumulate, tcgen05), f32 path code",
            "data": "synthetic (seeded terrain square)",
            "config": {"workload": "surrogate painter, terrain square 16 km^2: a step is one seeded 16x8 tile x one "
                                   f"1/{args.slices} slice of the 3.99 M sources", "l2": "flushed between painters",
                       "exact_within_m": exact_within_m},
            "exact_value": exact, "speedup_vs_exact": value / exact, "surrogate_share": taken / max(paths, 1),
            "path_error_db": {"p50": float(np.percentile(err, 50)), "p99": float(np.percentile(err, 99)),
                              "samples": int(err.size)},
            "cell_dba_error_db": {"p50": float(np.median(cell_err)), "p99": float(np.percentile(cell_err, 99)),
                                  "max": float(cell_err.max()), "mean_signed": float(cell_signed.mean())},
            "training": {"samples": int(n_train), "epochs": 6, "seconds": train_s, "loss": [float(v) for v in hist]},
            "clocks": clocks.summary(), "gpu_launches": args.steps * 5,
        }), flush=True)
    ctx.close()


def host_ndens(pixels, shares, runs, threads):
    """Nden of each packed pixel by the library's host composition (qm_pixel_ndens, equal to the
    FP64 oracle's composition bit for bit) on curves of the oracle's Zwicker in double, a host
    thread a pixel."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import oracle
    from quietmap_b200 import native

    def one(packed):
        at, n_layers = 0, 6
        for _ in range(n_layers):
            at += 4 + int(packed[at + 3]) * 43
        tables = np.zeros((n_layers + 1, 3, 191))
        for c in range(n_layers + 1):
            for p in range(3):
                shape = packed[at + (c * 3 + p) * 28: at + (c * 3 + p + 1) * 28].astype(np.float64)
                if not np.isnan(shape[0]):
                    tables[c, p] = oracle.zwicker_many(shape[None, :] + (-30.0 + np.arange(191))[:, None], nthreads=1)
        return native.pixel_ndens(packed, n_layers, 2.0, tables, shares, runs)
    with ThreadPoolExecutor(max_workers=threads) as pool:
        return np.array(list(pool.map(one, pixels)))


def loudness(args, rank, world, local):
    """Batch::loudness on the device: a step is one call of 8,192 packed pixels (the reference's
    batch, paint/src/exact.rs:21-22), 6 layers, the map's 2 dB grid, hours grouped 4/1/3 by 12
    hourly profiles; pixels/s of device time, and end to end through the C ABI with the pixels'
    upload and the Nden read back."""
    import torch
    from oracle import oracle
    from quietmap_b200 import native, scenes
    n = 8192
    pixels, shares, runs = scenes.loudness_pixels(n, seed=11 + rank)
    n_floats = sum(len(p) for p in pixels)
    ctx = native.Context(local if world > 1 else 0)
    torch.cuda.set_device(local if world > 1 else 0)
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    for _ in range(args.warmup):
        ctx.pixel_loudness(pixels, 6, 2.0, shares, runs)
    k_ms, wall = 0.0, 0.0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            got, ms = ctx.pixel_loudness(pixels, 6, 2.0, shares, runs, stats=True)
            wall += time.perf_counter() - t0
            k_ms += ms
    if rank == 0:
        line = {
            "metric": "Batch::loudness pixels/s (packed pixels to Nden per layer and place), 1 B200",
            "value": n * args.steps / (k_ms / 1e3), "unit": "pixels/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": k_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 distributions, f32 Zwicker", "data": "synthetic (seeded packed pixels)",
            "config": {"workload": f"{n} packed pixels a call (6 layers, 0-4 lines each: roads at mean flow, profiled "
                                   "roads, events, streams), 2 dB grid, hours in 4/1/3 groups of 12 profiles",
                       "floats_per_call": n_floats, "l2": "flushed between steps"},
            "e2e": {"value": n * args.steps / wall, "unit": "pixels/s", "h2d_bytes_per_step": n_floats * 4 + n * 8,
                    "d2h_bytes_per_step": n * 7 * 4 + n * 4},
            "clocks": clocks.summary(), "gpu_launches": args.steps,
        }
        if not args.no_cpu_baseline and world == 1:
            threads = oracle.threads()
            m = threads
            t0 = time.perf_counter()
            host_ndens(pixels[:m], shares, runs, threads)
            dt = time.perf_counter() - t0
            m = min(n, max(m, int(m * 12.0 / max(dt, 1e-3))))
            t0 = time.perf_counter()
            want = host_ndens(pixels[:m], shares, runs, threads)
            dt = time.perf_counter() - t0
            rel = np.abs(got[:m] - want) / np.maximum(np.abs(want), 1e-12)
            line["cpu_baseline"] = dict(value=m / dt, unit="pixels/s", cores=threads, kind="port",
                                        sample=f"the first {m} pixels by the host composition equal to the FP64 "
                                               f"oracle's, curves by the oracle's Zwicker ({dt:.1f} s)")
            line["parity"] = {"pixels": m, "max_relative_nden_error": float(rel[want != 0].max()),
                              "zero_where_host_zero": bool(np.all(got[:m][want == 0] == 0))}
        print(json.dumps(line), flush=True)
    ctx.close()


def flight_sums(args, rank, world, local):
    """Batch::flight_sums on the device: the flight workload's square (2000 flights x 50 segments over
    1024^2 cells at 100 m) summed into 400 m and 1,600 m boxes, asked at a lattice of points with their
    horizons (every aircraft tile within 16 km, its fine boxes within 3 km); a step is one call for
    every point."""
    import torch
    from quietmap_b200 import native, scenes
    world_boxes = scenes.flight_boxes_square(seed=3 + rank, n_flights=args.flights, receivers=args.cells_side)
    n = args.lattice_side
    xs = (np.arange(n) + 0.5) * world_boxes.side_m / n
    xy = np.stack(np.meshgrid(xs, xs), -1).reshape(-1, 2)
    points, hz, segs, n_sums = scenes.flight_requests(world_boxes, xy, seed=5 + rank)
    ctx = native.Context(local if world > 1 else 0)
    torch.cuda.set_device(local if world > 1 else 0)
    dev = ctx.flight_boxes(world_boxes.boxes)
    for _ in range(args.warmup):
        dev.sums(points, hz, segs, n_sums)
    torch.cuda.synchronize()
    k_ms, wall, reads, heard = 0.0, 0.0, 0, 0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            got, st = dev.sums(points, hz, segs, n_sums, stats=True)
            wall += time.perf_counter() - t0
            k_ms += st["kernel_ms"]
            reads += st["box_reads"]
            heard += st["boxes_heard"]
    if rank == 0:
        n_pts = len(points)
        line = {
            "metric": "Batch::flight_sums points/s (aircraft boxes within 16 km summed with pass classes), 1 B200",
            "value": n_pts * args.steps / (k_ms / 1e3), "unit": "points/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": k_ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded flights, NPD tables and horizons)",
            "config": {"workload": f"{n}^2 lattice points over the {args.cells_side * 0.1:.1f} km square of "
                                   f"{args.flights} flights x 50 segments, {len(world_boxes.boxes)} boxes",
                       "box_reads_per_step": reads // args.steps, "boxes_heard_per_step": heard // args.steps,
                       "l2": "boxes resident (the square's boxes are decoded once and read by every point)"},
            "box_reads_per_s": reads / (k_ms / 1e3), "boxes_heard_per_s": heard / (k_ms / 1e3),
            "e2e": {"value": n_pts * args.steps / wall, "unit": "points/s",
                    "h2d_bytes_per_step": points.nbytes + hz.nbytes + segs.nbytes,
                    "d2h_bytes_per_step": n_sums * abi_flight_sums() * 8},
            "clocks": clocks.summary(), "gpu_launches": args.steps,
        }
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle
            threads = oracle.threads()
            m = 8
            pick = np.random.default_rng(43).permutation(n_pts)
            for _ in range(2):
                mine = np.isin(segs["point"], pick[:m])
                t0 = time.perf_counter()
                want, _ = oracle.flight_sums(world_boxes.boxes, points, hz, segs[mine], n_sums, threads)
                dt = time.perf_counter() - t0
                if dt > 6.0 or m >= n_pts:
                    break
                m = min(n_pts, max(m, int(m * 12.0 / max(dt, 1e-3))))
            rows = np.concatenate([2 * pick[:m], 2 * pick[:m] + 1])
            scale = np.maximum(np.abs(want[rows]), 1e-300)
            rel = np.where(want[rows] != 0.0, np.abs(got[rows] - want[rows]) / scale, np.abs(got[rows]))
            line["cpu_baseline"] = dict(value=m / dt, unit="points/s", cores=threads, kind="port",
                                        sample=f"{m} of the lattice's points, every box they hear ({dt:.1f} s)")
            line["parity"] = {"points": m, "max_relative_error": float(rel.max())}
        print(json.dumps(line), flush=True)
    dev.close()
    ctx.close()


def horizons(args, rank, world, local):
    """The points' horizons for aircraft screening on the device (Horizons::build, which the
    reference runs on the cores for every flight request): the terrain square (16 km^2, fBm DEM,
    30,000 buildings), a step builds a 64^2 lattice of points' horizons (32 terrain sectors x 48
    samples, 256 building rays of 512 m each)."""
    import torch
    from quietmap_b200 import native, scenes
    scene, _ = scenes.terrain_square()
    ext = np.array(scene.extent_steps, dtype=np.float64)
    n = args.lattice_side
    xs = (np.arange(n) + 0.5) / n
    xy = np.stack(np.meshgrid(xs * ext[0], xs * ext[1]), -1).reshape(-1, 2)
    ctx = native.Context(local if world > 1 else 0)
    torch.cuda.set_device(local if world > 1 else 0)
    dev = ctx.scene(scene)
    alt = np.full(len(xy), 4.0) + scenes_ground(scene, xy)
    own = np.zeros(len(xy), np.uint64)
    for _ in range(args.warmup):
        dev.flight_horizons(xy, alt, own)
    k_ms, wall = 0.0, 0.0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            got, ms = dev.flight_horizons(xy, alt, own, stats=True)
            wall += time.perf_counter() - t0
            k_ms += ms
    if rank == 0:
        pts = len(xy)
        line = {
            "metric": "receiver horizons/s for aircraft screening (Horizons::build), 1 B200", "value": pts * args.steps / (k_ms / 1e3),
            "unit": "points/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": k_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded terrain square)",
            "config": {"workload": f"{n}^2 lattice points over the terrain square (16 km^2, 30,000 buildings): "
                                   "32 terrain sectors x 48 samples and 256 building rays of 512 m a point"},
            "e2e": {"value": pts * args.steps / wall, "unit": "points/s", "h2d_bytes_per_step": pts * 28,
                    "d2h_bytes_per_step": int(got.nbytes)},
            "clocks": clocks.summary(), "gpu_launches": args.steps,
        }
        line["flight_sums_on_scene"] = flight_sums_on_scene(args, rank, ctx, dev, scene, xy, alt, own)
        if not args.no_cpu_baseline and world == 1:
            from oracle import oracle
            ora = oracle.OracleScene(scene)
            threads = oracle.threads()
            m = len(xy)  # the whole lattice: a fraction of a second on 16 threads
            t0 = time.perf_counter()
            want = ora.flight_horizons(xy[:m], alt[:m], own[:m], threads)
            dt = time.perf_counter() - t0
            same = bool(np.array_equal(np.nan_to_num(got[:m], nan=7.0, neginf=-7.0),
                                       np.nan_to_num(want, nan=7.0, neginf=-7.0)))
            line["cpu_baseline"] = dict(value=m / dt, unit="points/s", cores=threads, kind="port",
                                        sample=f"the lattice's {m} points ({dt:.2f} s)")
            line["parity"] = {"points": m, "bit_identical": same}
        print(json.dumps(line), flush=True)
    dev.close()
    ctx.close()


def flight_sums_on_scene(args, rank, ctx, dev, scene, xy, alt, own):
    """Batch::flight_sums for the lattice's points end to end, their horizons built on the device
    and read there (qm_flight_sums_on_scene), against the same sums through two calls: the horizons
    down to the host (qm_scene_flight_horizons) and up again with the requests (qm_flight_sums).
    The boxes are the flight workload's (2000 flights over the 102.4 km square); the points hear
    every aircraft tile within 16 km of the terrain square's corner of it."""
    from quietmap_b200 import scenes
    world_boxes = scenes.flight_boxes_square(seed=3 + rank, n_flights=args.flights, receivers=args.cells_side)
    points, _, segs, n_sums = scenes.flight_requests(world_boxes, xy * scene.step_m, horizons=False, seed=5 + rank)
    points["altitude_m"] = alt
    boxes = ctx.flight_boxes(world_boxes.boxes)
    for _ in range(args.warmup):
        boxes.sums_on_scene(dev, points, own, segs, n_sums)
    one = two = 0.0
    worst = 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        a = boxes.sums_on_scene(dev, points, own, segs, n_sums)
        one += time.perf_counter() - t0
        t0 = time.perf_counter()
        hz = dev.flight_horizons(xy, alt, own)
        b = boxes.sums(points, hz.reshape(-1), segs, n_sums)
        two += time.perf_counter() - t0
        rel = np.where(b != 0.0, np.abs(a - b) / np.maximum(np.abs(b), 1e-300), np.abs(a))
        worst = max(worst, float(rel.max()))
    boxes.close()
    pts = len(points)
    return {"value": pts * args.steps / one, "unit": "points/s", "two_calls_value": pts * args.steps / two,
            "speedup_vs_two_calls": two / one, "box_reads_per_step": int(segs["count"].sum()),
            "horizon_bytes_kept_on_device_per_step": 2 * int(hz.nbytes),
            "h2d_bytes_per_step": int(points.nbytes + segs.nbytes + pts * 28),
            "d2h_bytes_per_step": int(n_sums * abi_flight_sums() * 8),
            "max_relative_difference_vs_two_calls": worst}


def scenes_ground(scene, xy):
    """The ground (m) under lattice positions of a scene: its DEM bilinear, or its flat ground."""
    if scene.dem_altitude is None:
        return np.full(len(xy), scene.flat_altitude_m if hasattr(scene, "flat_altitude_m") else 0.0)
    z = np.asarray(scene.dem_altitude, dtype=np.float64)
    sp, ox, oy = scene.dem_spacing, scene.dem_origin[0], scene.dem_origin[1]
    fx = np.clip((xy[:, 0] - ox) / sp, 0, z.shape[1] - 1)
    fy = np.clip((xy[:, 1] - oy) / sp, 0, z.shape[0] - 1)
    i0 = np.minimum(np.floor(fx).astype(int), z.shape[1] - 2)
    j0 = np.minimum(np.floor(fy).astype(int), z.shape[0] - 2)
    ax, ay = fx - i0, fy - j0
    lo = z[j0, i0] + ax * (z[j0, i0 + 1] - z[j0, i0])
    hi = z[j0 + 1, i0] + ax * (z[j0 + 1, i0 + 1] - z[j0 + 1, i0])
    return lo + ay * (hi - lo)


def abi_flight_sums():
    from quietmap_b200 import abi
    return abi.FLIGHT_SUMS


def tile_batch(args, rank, world, local):
    """Uneven tiles (config 4): 4096 tiles, sides log-uniform 32-512 receivers at 7.8125 m, each with
    its own road segments (log-uniform 10-50,000) and buildings (log-uniform 0-20,000) drawn in a
    region of its own; a step paints a seeded batch of `--tiles` of them as one autotuned,
    graph-captured persistent launch per thread count. A tile paints every receiver against its
    first roads up to 2^26 paths (a prefix of independent draws). Beside it: the same batch with
    the default launch shape, and one qm_paint_grid call per tile."""
    import torch
    from quietmap_b200 import native, scenes
    specs = scenes.uneven_tile_specs(n_tiles=4096)
    rng = np.random.default_rng(7 + rank)
    pick = sorted(rng.choice(len(specs), args.tiles, replace=False))
    world_scene, tiles = scenes.uneven_tile_world([specs[k] for k in pick], max_paths_per_tile=1 << 26)
    cells = sum(t["nx"] * t["ny"] for t in tiles)
    paths = sum(t["nx"] * t["ny"] * (t["source_end"] - t["source_begin"]) for t in tiles)
    ctx = native.Context(local if world > 1 else 0)
    dev = ctx.scene(world_scene)
    # Autotuner: two sample tiles per size bucket from the batch.
    sample, per = [], {}
    for t in tiles:
        b = native.tile_bucket(t)
        if per.get(b, 0) < 2:
            sample.append(t)
            per[b] = per.get(b, 0) + 1
    t0 = time.perf_counter()
    table, timings = native.autotune(dev, sample)
    tune_s = time.perf_counter() - t0
    plan = native.BatchPlan(dev, tiles, table=table)
    for _ in range(args.warmup):
        plan.run()
    flush = torch.empty(64 << 20, dtype=torch.float32, device="cuda")
    ms = 0.0
    with ClockSampler(local) as clocks:
        for _ in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            ms += plan.run()["kernel_ms"]
    _, dba_batch, _ = plan.read()
    plan.close()
    default = native.BatchPlan(dev, tiles)
    default_ms = default.run()["kernel_ms"]
    default.close()
    one_ms, one_wall = 0.0, time.perf_counter()
    dba_one = np.empty(cells, np.float32)
    for t in tiles:
        g = scenes.Grid(origin=t["origin"], spacing=t["spacing"], nx=t["nx"], ny=t["ny"],
                        source_begin=t["source_begin"], source_end=t["source_end"])
        _, d, _, _, st = dev.paint_grid(g, histogram=False)
        dba_one[t["cell_offset"]:t["cell_offset"] + g.cells] = d
        one_ms += st["kernel_ms"]
    one_wall = time.perf_counter() - one_wall
    if rank == 0:
        per_step_s = ms / 1e3 / args.steps
        cfg = [dict(block=f"{table.bucket[b].block_w}x{table.bucket[b].block_h}", threads=table.bucket[b].threads,
                    chunk=table.bucket[b].chunk) for b in range(4)]
        print(json.dumps({
            "metric": "cells/s and receiver-source paths/s of a batch of uneven tiles, 1 B200",
            "value": paths / per_step_s, "unit": "paths/s", "cells_per_s": cells / per_step_s,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded tiles, each its own roads and buildings)",
            "config": {"workload": f"{args.tiles} of 4096 uneven tiles (sides log-uniform 32-512 receivers at "
                                   "7.8125 m; each its own roads, log-uniform 10-50,000 segments at 1 m points, and "
                                   "buildings, log-uniform 0-20,000 rectangles, in a region of its own; a tile's "
                                   f"paths capped at 2^26 by a prefix of its roads): {cells} cells, {paths} paths per "
                                   "step, one autotuned persistent launch per thread count, CUDA graph",
                       "buildings": sum(t["buildings"] for t in tiles),
                       "segments_kept": sum(t["kept_segments"] for t in tiles),
                       "l2": "flushed between steps", "tuned": cfg, "autotune_s": tune_s},
            "default_shape_paths_per_s": paths / (default_ms / 1e3),
            "one_call_per_tile": {"paths_per_s_device": paths / (one_ms / 1e3), "paths_per_s_wall": paths / one_wall,
                                  "cells_per_s_wall": cells / one_wall},
            "batch_vs_one_call_dba_max_diff_db": float(np.max(np.abs(dba_batch - dba_one))),
            "clocks": clocks.summary(), "gpu_launches": args.steps * 3,
        }), flush=True)
    ctx.close()


def reference_arm(args, rank, world):
    """The reference's CPU path (its FP64 restatement) on all host threads, rank 0 only, on the
    same workload and the same sample rule as the GPU arm's CPU baseline: the receivers of the GPU
    arm's first timed step against a stratified, seeded subsample of that step's source slice."""
    if rank != 0:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()
        return
    workload_name = "terrain" if args.workload not in ("terrain", "road") else args.workload
    scene, steps, desc = workload(workload_name, 0, args.slices, args.sources)
    g = steps[args.warmup % len(steps)][0]
    # Warm-up: the sample is sized here (untimed), then each timed step runs it once.
    ora, grid, idx, threads = cpu_sample(scene, g, seconds=8.0)
    times = [cpu_run(ora, grid, threads) for _ in range(max(args.steps, 1))]
    dt = float(np.median(times))
    value = grid.cells * len(idx) / dt
    line = {
        "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator of the workload's geometry)",
        "config": dict(desc, parallelism="host threads"), "impl": "reference",
        "cpu_baseline": dict(value=value, unit="paths/s", cores=threads, kind="port",
                             sample=cpu_description(grid, g, idx, dt) + " per step"),
        "per_path": cpu_work(ora, scene, grid, idx),
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
