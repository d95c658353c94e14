"""Benchmark of the exact painter: receiver-source paths per second on one B200.

Workload (default `terrain`): the 16 km^2 terrain square at full size (fBm DEM at 5 m posts, Voronoi
ground factor, 20,000 road and rail segments as ~4.0 M one-metre point sources, 30,000 polygon
buildings, favourable probability 0.5), painted for a seeded sample of receiver tiles of the
2048 x 2048 grid against every source. A step paints one sample block of receivers.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload terrain|road]

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
FP32_NOMINAL_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="terrain", choices=["terrain", "road"])
    ap.add_argument("--receivers", type=int, default=0, help="receivers per step (0: workload default)")
    ap.add_argument("--sources", type=int, default=0,
                    help="paint only the first N sources (a small case for profiling; 0: all)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload(name, rank, receivers):
    from quietmap_b200 import scenes
    if name == "road":
        scene, full = scenes.road_square()
        if not receivers:
            desc = dict(workload="road square 1 km, 128x128 receivers x 77k point sources (flat, G=0.5, "
                                 "homogeneous)", global_batch=full.cells)
            return scene, [full], desc
    else:
        scene, full = scenes.terrain_square()
    per_step = receivers or 256
    tile_w, tile_h = 16, 8
    n_tiles = max(per_step // (tile_w * tile_h), 1)
    rng = np.random.default_rng(1000 + rank)
    blocks = []
    for _ in range(64):
        tiles = []
        for _ in range(n_tiles):
            tx = int(rng.integers(0, full.nx // tile_w))
            ty = int(rng.integers(0, full.ny // tile_h))
            tiles.append((tx, ty))
        blocks.append(tiles)
    grids = []
    for tiles in blocks:
        # One grid per tile; a step paints all tiles of its block.
        grids.append([scenes.Grid(origin=(full.origin[0] + tx * tile_w * full.spacing,
                                          full.origin[1] + ty * tile_h * full.spacing),
                                  spacing=full.spacing, nx=tile_w, ny=tile_h) for tx, ty in tiles])
    if name == "road":
        what = "road square 1 km (128^2 grid at 7.8125 m, flat G=0.5, homogeneous), 300 buildings"
    else:
        what = "terrain square 16 km^2 (2048^2 grid at 1.953 m), 30,000 buildings, fBm DEM"
    desc = dict(workload=f"{what}: {n_tiles} seeded 16x8 receiver tiles per step x {len(scene.sources)} "
                         f"point sources", global_batch=n_tiles * tile_w * tile_h)
    return scene, grids, desc


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
                "reasons": reasons}


def cpu_baseline(scene, grid_list, seconds=12.0):
    """The FP64 oracle on all host threads: paths/s on a bounded sample (one receiver of the first
    tile against a prefix of the sources, grown until it takes about `seconds`)."""
    from oracle import oracle
    from quietmap_b200 import scenes
    ora = oracle.OracleScene(scene)
    g0 = grid_list[0][0] if isinstance(grid_list[0], list) else grid_list[0]
    threads = oracle.threads()
    n = 2000
    while True:
        grid = scenes.Grid(origin=g0.origin, spacing=g0.spacing, nx=1, ny=1, source_begin=0,
                           source_end=min(n, len(scene.sources)))
        t0 = time.perf_counter()
        ora.paint_grid(grid, nthreads=threads)
        dt = time.perf_counter() - t0
        if dt > seconds / 4 or n >= len(scene.sources):
            break
        n = min(int(n * max(2.0, seconds / 4 / max(dt, 1e-3))), len(scene.sources))
    # Spread the sample over threads: several receivers of the tile, the same source prefix.
    k = max(1, min(threads, 8))
    grid = scenes.Grid(origin=g0.origin, spacing=g0.spacing, nx=k, ny=1, source_begin=0, source_end=n)
    t0 = time.perf_counter()
    ora.paint_grid(grid, nthreads=threads)
    dt = time.perf_counter() - t0
    return dict(value=k * n / dt, unit="paths/s", cores=threads, kind="port",
                sample=f"{k} receivers x first {n} point sources ({k * n} paths, {dt:.1f} s)")


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
    import torch
    from quietmap_b200 import native
    scene, grids, desc = workload(args.workload, rank, args.receivers)
    ctx = native.Context(local if world > 1 else 0)
    dev = ctx.scene(scene)
    n_src = len(scene.sources)

    if args.sources:
        for block in grids:
            for g in (block if isinstance(block, list) else [block]):
                g.source_begin, g.source_end = 0, min(args.sources, n_src)
        desc["workload"] += f" (first {min(args.sources, n_src)} sources only)"

    def step(i):
        block = grids[i % len(grids)]
        tiles = block if isinstance(block, list) else [block]
        paths, kms, crossings = 0, 0.0, 0
        for g in tiles:
            _, _, _, _, st = dev.paint_grid(g)
            paths += st["paths"]
            kms += st["kernel_ms"]
            crossings += st["crossings"]
            for k in ("edge_tests", "vertices", "candidates"):
                work[k] += st[k]
        return paths, kms, crossings, len(tiles)

    work = dict(edge_tests=0, vertices=0, candidates=0)

    for i in range(args.warmup):
        step(i)
    work.update(edge_tests=0, vertices=0, candidates=0)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    total_paths, total_ms, total_cross, calls = 0, 0.0, 0, 0
    with ClockSampler(local) as clocks:
        t0 = time.perf_counter()
        for i in range(args.steps):
            p, k, c, n = step(args.warmup + i)
            total_paths += p
            total_ms += k
            total_cross += c
            calls += n
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
    if world > 1:
        t = torch.tensor([total_ms, wall], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms, wall = float(t[0]), float(t[1])
        tp = torch.tensor([total_paths], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(tp)
        total_paths = int(tp[0])
    if rank == 0:
        value = total_paths / (total_ms / 1e3)
        e2e = total_paths / wall
        cells_per_call = grids[0][0].cells if isinstance(grids[0], list) else grids[0].cells
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "paths/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 (f64 for path differences and crossing chainage)",
            "data": "synthetic (seeded generator of the workload's geometry)",
            "config": dict(desc, sources=n_src, parallelism=f"replicas x{world}",
                           l2="inputs larger than L2 (sources 511 MB resident)"),
            "e2e": {"value": e2e, "unit": "paths/s",
                    "h2d_bytes_per_step": calls * cells_per_call * 8 // args.steps if args.steps else 0,
                    "d2h_bytes_per_step": calls * (cells_per_call * 40 + 1800 * 4) // args.steps if args.steps else 0},
            "gpu_launches": calls * 2,
            "clocks": clocks.summary(),
            "per_path": dict(crossings=total_cross / max(total_paths, 1),
                             **{k: v / max(total_paths, 1) for k, v in work.items()}),
        }
        if not args.no_cpu_baseline and world == 1:
            line["cpu_baseline"] = cpu_baseline(scene, grids)
        print(json.dumps(line), flush=True)
    dev.close()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def reference_arm(args, rank, world):
    """The reference's CPU path (its FP64 restatement) on all host threads, rank 0 only."""
    if rank != 0:
        if world > 1:
            import torch.distributed as tdist
            tdist.destroy_process_group()
        return
    scene, grids, desc = workload(args.workload, 0, args.receivers)
    base = None
    for _ in range(args.warmup):
        pass
    samples = []
    for _ in range(max(args.steps, 1)):
        base = cpu_baseline(scene, grids, seconds=8.0)
        samples.append(base["value"])
    value = float(np.median(samples))
    line = {
        "metric": METRIC, "value": value, "unit": "paths/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded generator of the workload's geometry)",
        "config": dict(desc, parallelism="host threads"), "impl": "reference",
        "cpu_baseline": dict(base, value=value),
        "e2e": {"value": value, "unit": "paths/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as tdist
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
