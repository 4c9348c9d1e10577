#!/usr/bin/env python3
"""Closest-hit cast benchmark: Mrays/s on a 1,048,576-triangle displaced sphere.

Workload (one "step"): 16,777,216 rays, origins uniform in [-2, 2]^3, directions uniform on
the sphere, min_t 0, max_t Ray_max_t, cast closest-hit against the SAH BVH of a tetra-sphere
(n = 512) displaced by fBm of amplitude 0.1 (6 octaves, seed 1).  Rays (512 MiB) exceed
the 126 MB L2, so no flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sprout|reference]

Multi-GPU (torchrun, one process per GPU): every rank casts its own 16,777,216 rays (ray
indices rank*R .. rank*R+R-1) against its own copy of the tree; no collective touches the
data path (weak scaling).  NCCL carries only the barrier and the max-over-ranks time.

Prints one JSON line (rank 0).
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import pathlib
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

MESH_N = 512
RAYS = 1 << 24
SEED = 1
ALGO_BYTES_PER_RAY = 40  # 32 B ray in + 4 B id + 4 B t out
METRIC = "Mrays/s closest-hit"
WORKLOAD = "cast: 1,048,576-tri fBm-displaced tetra-sphere (n=512, amp 0.1, seed 1), 16,777,216 rays o~U[-2,2]^3 d~S^2 (seed 1)"


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=50)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=["sprout", "reference"], default="sprout")
    p.add_argument("--rays", type=int, default=RAYS)
    p.add_argument("--mesh-n", type=int, default=MESH_N)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-render", action="store_true", help="skip the path-tracer measurement")
    p.add_argument("--render-spp", type=int, default=64)
    p.add_argument("--no-wavefront", action="store_true",
                   help="skip the 1920x1080 many-instances, many-lights render measurement")
    p.add_argument("--no-volume", action="store_true",
                   help="skip the 64-view heterogeneous-volume render measurement")
    p.add_argument("--no-guiding", action="store_true",
                   help="skip the doorway time-to-relMSE measurement (plain MIS against path guiding)")
    return p.parse_args()


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes per ray of the closest-hit kernel, from the committed ncu summary."""
    f = ROOT / "profiles" / "cast_closest_hit_ncu.txt"
    if not f.exists():
        return None
    m = re.search(r"dram_bytes_per_ray:\s*([0-9.eE+-]+)", f.read_text())
    return float(m.group(1)) if m else None


CLOCK_SAMPLER = r"""
import sys, time
import pynvml
pynvml.nvmlInit()
entry = sys.argv[1]
h = (pynvml.nvmlDeviceGetHandleByUUID(entry) if entry.startswith("GPU-")
     else pynvml.nvmlDeviceGetHandleByIndex(int(entry)))
print("max", pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM), flush=True)
while True:
    mhz = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
    bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
    print(f"{time.monotonic():.6f} {mhz} {bits}", flush=True)
    time.sleep(0.002)
"""


class ClockSampler:
    """SM clock and clock-event (throttle) reasons read through NVML every 2 ms by a separate
    process (read-only queries; no setting changes); mark() brackets the timed region and
    summary() keeps the samples taken inside it."""

    REASONS = {
        "hw_slowdown": 0x8,
        "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40,
        "hw_power_brake": 0x80,
        "sw_power_cap": 0x4,
    }

    def __init__(self, gpu_index: int):
        visible = [v.strip() for v in os.environ.get("CUDA_VISIBLE_DEVICES", "").split(",") if v.strip()]
        self.entry = visible[gpu_index] if gpu_index < len(visible) else str(gpu_index)
        self.proc = None
        self.lines = []
        self.max_mhz = None
        self.t0 = self.t1 = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", CLOCK_SAMPLER, self.entry],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
            deadline = time.monotonic() + 20.0
            while len(self.lines) < 3 and time.monotonic() < deadline and self.proc.poll() is None:
                time.sleep(0.01)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.split())

    def mark_start(self):
        self.t0 = time.monotonic()

    def mark_end(self):
        self.t1 = time.monotonic()
        time.sleep(0.01)

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        samples = []
        for parts in self.lines:
            if parts and parts[0] == "max":
                self.max_mhz = int(parts[1])
            elif len(parts) == 3:
                t, mhz, bits = float(parts[0]), int(parts[1]), int(parts[2])
                if self.t0 is not None and self.t0 <= t <= (self.t1 or t):
                    samples.append((mhz, bits))
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"], "samples": 0}
        seen = sorted({name for _, bits in samples for name, mask in self.REASONS.items() if bits & mask})
        return {"sm_mhz": statistics.median(m for m, _ in samples), "sm_max_mhz": self.max_mhz,
                "reasons": seen, "samples": len(samples), "source": "NVML in a separate process, 2 ms period"}


def rank_rays(rank: int, count: int) -> np.ndarray:
    """This rank's share of the workload: rays rank*count .. rank*count+count-1 of the seeded
    stream (every ray's stream depends only on its index, so N ranks together cast the first
    N*count rays of one sequence -- weak scaling with disjoint ranges)."""
    import sprout_b200 as sb

    return sb.random_rays(count, seed=SEED, first=rank * count)


def max_over_ranks(value: float, dist, device) -> float:
    """The slowest rank's time (the job's time); value itself without a process group."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def reference_run(mesh_path, rays_path, steps, warmup, num_rays=None):
    """Times the reference's Builder_SAH + Tree::intersect (oracle/_ref/ref_cast) on all host
    threads over warmup + steps passes; with num_rays also returns its ids and t (last pass)."""
    import oracle

    with tempfile.TemporaryDirectory() as tmp:
        out = os.path.join(tmp, "out.bin")
        res = subprocess.run([str(oracle.REF_CAST), mesh_path, rays_path, out, "0", "hit", str(steps + warmup)],
                             capture_output=True, text=True, check=True)
        timing = json.loads(res.stdout.strip().splitlines()[-1])
        if num_rays is None:
            return timing
        raw = np.fromfile(out, np.uint8, count=8 * num_rays)
    return timing, raw[: 4 * num_rays].view(np.uint32), raw[4 * num_rays:].view(np.float32)


def write_inputs(tmp, pos, idx, rays):
    import oracle

    mesh_path = os.path.join(tmp, "mesh.bin")
    rays_path = os.path.join(tmp, "rays.bin")
    oracle.write_mesh(mesh_path, pos, idx)
    oracle.write_rays(rays_path, rays)
    return mesh_path, rays_path


def workload_config(rays: int, triangles: int, world: int) -> dict:
    """The config object both arms print (same keys and values for the same workload)."""
    return {"workload": WORKLOAD, "rays_per_step_per_gpu": rays, "triangles": triangles,
            "parallelism": f"replicas x{world} (independent ray ranges)",
            "l2": "inputs (rays, 512 MiB) larger than L2; no flush"}


def l2_copy_bandwidth(torch) -> float:
    """L2-resident copy bandwidth in GB/s (bytes read + written): torch copy_ between two
    32 MiB buffers (together well inside the 126 MB L2), 64 copies replayed from one CUDA
    graph, best of 5 replays timed with CUDA events."""
    n = (32 << 20) // 4
    a = torch.ones(n, dtype=torch.float32, device="cuda")
    b = torch.empty_like(a)
    reps = 64
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream().wait_stream(side)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(reps):
            b.copy_(a)
    best = float("inf")
    for _ in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        graph.replay()
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del graph
    return 2 * 4 * n * reps / best / 1e9


def cpu_lscpu():
    try:
        out = subprocess.run(["lscpu"], capture_output=True, text=True).stdout
        m = re.search(r"Model name:\s*(.+)", out)
        return m.group(1).strip() if m else "unknown"
    except OSError:
        return "unknown"


def run_reference_arm(args, world, rank):
    """The reference's own CPU traversal (Builder_SAH(16,64,4) + Tree::intersect, compiled
    from its sources into oracle/_ref/ref_cast) on all host threads.  The inputs come from the
    oracle's C restatement of the benchmark synthesis, so this arm loads no product code."""
    if rank != 0:
        return
    import oracle

    if not oracle.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_cast not built"}))
        return
    pos, idx = oracle.synth_sphere_mesh(args.mesh_n, 0.1, SEED)
    rays = oracle.synth_rays(args.rays, seed=SEED)
    with tempfile.TemporaryDirectory() as tmp:
        mesh_path, rays_path = write_inputs(tmp, pos, idx, rays)
        del rays
        timing = reference_run(mesh_path, rays_path, args.steps, args.warmup)
    times = timing["hit_s_list"][args.warmup:]
    total = sum(times)
    value = args.rays * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s",
        "n_gpus": world, "steps": len(times), "warmup": args.warmup,
        "ms_per_step": round(1e3 * total / len(times), 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.rays, int(idx.shape[0]), world),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": timing["threads"],
                         "kind": "reference", "cpu": cpu_lscpu(),
                         "sample": f"full workload ({args.rays} rays) per step, reference Builder_SAH(16,64,4) "
                                   f"tree (build {timing['build_s']:.3f} s, untimed) + Tree::intersect; inputs "
                                   f"from the oracle's restatement of the benchmark synthesis"},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def measure_render(args, with_cpu):
    """Plain MIS path tracing through the su_* C API: the Cornell scene (512x512, 64 spp, with
    time to relMSE 0.01), the many-instances, many-lights scene (1920x1080, 256 spp, depth 12;
    one warm-up frame, one timed frame), the heterogeneous volume (64 views, 128 spp; and the
    spectral mode's phase guiding against plain on its first view) and the doorway interior's
    time to relMSE 0.01, plain MIS against learned guiding (1280x720)."""
    from sprout_b200 import render_bench

    out = {"cornell": render_bench.measure("cornell", spp=args.render_spp, frames=3, convergence=True,
                                           cpu_reference=with_cpu)}
    if not args.no_wavefront:
        out["wavefront"] = render_bench.measure("wavefront", frames=1, cpu_reference=with_cpu)
        out["wavefront_flat"] = render_bench.measure("wavefront_flat", frames=1)
    if not args.no_volume:
        out["volume"] = render_bench.measure_volume(views=64, spp=128, cpu_reference=with_cpu)
        out["volume"]["phase_guiding"] = render_bench.measure_phase_guiding(fractions=(0.1, 0.25))
    if not args.no_guiding:
        out["guiding"] = render_bench.measure_guiding()
    return out


def main():
    args = parse_args()
    world, rank, local = dist_setup()
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return

    import torch

    import sprout_b200 as sb

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    pos, idx = sb.sphere_mesh(args.mesh_n, 0.1, SEED)
    rays_host = rank_rays(rank, args.rays)

    tree = sb.Tree()
    tree.build(pos, idx)
    info = tree.info()

    stream = torch.cuda.current_stream()
    d_rays = torch.from_numpy(rays_host).cuda()
    d_ids = torch.empty(args.rays, dtype=torch.int32, device="cuda")
    d_t = torch.empty(args.rays, dtype=torch.float32, device="cuda")

    for _ in range(args.warmup):
        tree.intersect(d_rays, out=(d_ids, d_t, None))
    barrier()

    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    with ClockSampler(local) as clocks:
        barrier()
        clocks.mark_start()
        t_begin = torch.cuda.Event(enable_timing=True)
        t_end = torch.cuda.Event(enable_timing=True)
        t_begin.record(stream)
        for k in range(args.steps):
            starts[k].record(stream)
            tree.intersect(d_rays, out=(d_ids, d_t, None))
            ends[k].record(stream)
        t_end.record(stream)
        barrier()
        clocks.mark_end()
    elapsed = max_over_ranks(t_begin.elapsed_time(t_end) / 1e3, dist, "cuda")
    kernel_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    assert tree.status() == 0

    hit_fraction = float((d_ids != -1).float().mean().item())
    gpu_ids = d_ids.cpu().numpy().view(np.uint32)
    gpu_t = d_t.cpu().numpy()

    # Work per ray (untimed counting pass) and the L2-resident copy bandwidth it is held against.
    steps_count = tree.traversal_stats(d_rays)
    l2_peak = l2_copy_bandwidth(torch)

    # any-hit throughput (reported beside the headline)
    d_occ = torch.empty(args.rays, dtype=torch.uint8, device="cuda")
    for _ in range(2):
        tree.intersect_p(d_rays, out=d_occ)
    a0 = torch.cuda.Event(enable_timing=True)
    a1 = torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    for _ in range(args.steps):
        tree.intersect_p(d_rays, out=d_occ)
    a1.record(stream)
    torch.cuda.synchronize()
    any_hit_mrays = args.rays * args.steps / (a0.elapsed_time(a1) / 1e3) / 1e6

    # end to end through the host-pointer entry point: pinned rays in, ids + t out
    e2e = None
    if not args.no_e2e:
        h_rays = torch.from_numpy(rays_host).pin_memory()
        h_ids = torch.empty(args.rays, dtype=torch.int32).pin_memory()
        h_t = torch.empty(args.rays, dtype=torch.float32).pin_memory()
        out = (h_ids.numpy().view(np.uint32), h_t.numpy(), None)
        rays_np = h_rays.numpy()
        for _ in range(2):
            tree.intersect(rays_np, out=out)
        barrier()
        e_steps = max(3, args.steps // 2)
        t0 = time.perf_counter()
        for _ in range(e_steps):
            tree.intersect(rays_np, out=out)
        e_el = max_over_ranks(time.perf_counter() - t0, dist, "cuda")
        e2e = {"value": round(world * args.rays * e_steps / e_el / 1e6, 3), "unit": "Mrays/s",
               "h2d_bytes_per_step": 32 * args.rays, "d2h_bytes_per_step": 8 * args.rays,
               "steps": e_steps, "path": "spb_intersect_host (pinned host buffers, 2-stream chunked copies)"}

    value = world * args.rays * args.steps / elapsed / 1e6
    mean_kernel_s = statistics.mean(kernel_ms) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = ALGO_BYTES_PER_RAY * args.rays / mean_kernel_s / 1e9
    traffic_per_ray = profiled_traffic()

    fetched_per_ray = (80.0 * steps_count["node_steps"] + 48.0 * steps_count["triangle_steps"]) / args.rays
    l2_achieved = fetched_per_ray * args.rays / mean_kernel_s / 1e9

    cpu_baseline = None
    id_parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        if oracle.reference_available():
            with tempfile.TemporaryDirectory() as tmp:
                mesh_path, rays_path = write_inputs(tmp, pos, idx, rays_host)
                timing, ref_ids, ref_t = reference_run(mesh_path, rays_path, 2, 1, num_rays=args.rays)
            t_cpu = statistics.mean(timing["hit_s_list"][1:])
            cpu_baseline = {"value": round(args.rays / t_cpu / 1e6, 3), "unit": "Mrays/s",
                            "cores": timing["threads"], "kind": "reference", "cpu": cpu_lscpu(),
                            "sample": f"full workload ({args.rays} rays), reference Builder_SAH(16,64,4) + "
                                      f"Tree::intersect on all host threads, mean of 2 passes (tree build "
                                      f"{timing['build_s']:.3f} s excluded)"}
            # Every ray of the timed cast against the reference's own answer for it.
            id_parity = oracle.id_parity(pos, idx, rays_host, ref_ids, ref_t, gpu_ids, gpu_t)
            id_parity["against"] = ("reference Builder_SAH(16,64,4) + Tree::intersect (oracle/_ref/ref_cast), "
                                    "every ray of the timed step")
            id_parity["explained_fraction"] = round(id_parity["explained_edge_tie"] / args.rays, 9)

    render = None
    if rank == 0 and not args.no_render:
        render = measure_render(args, with_cpu=(world == 1 and not args.no_cpu_baseline))

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * elapsed / args.steps, 4),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config(args.rays, info["num_triangles"], world),
            "tree": {"bvh_nodes": info["num_nodes"], "bvh_depth": info["max_depth"],
                     "build_s": round(info["build_seconds"], 3), "hit_fraction": round(hit_fraction, 5)},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 2), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 5), "peak_kind": peak_kind,
                         "algorithmic_bytes_per_ray": ALGO_BYTES_PER_RAY,
                         "kernel_ms_mean": round(1e3 * mean_kernel_s, 4),
                         "traffic": (round(traffic_per_ray * args.rays) if traffic_per_ray else None),
                         "note": "HBM carries only rays and results; the bound that matters is the "
                                 "node and triangle fetch below",
                         "l2": {"bound": "l2", "unit": "GB/s",
                                "achieved": round(l2_achieved, 1), "peak": round(l2_peak, 1),
                                "frac": round(l2_achieved / l2_peak, 4),
                                "peak_kind": "measured in this run: L2-resident copy bandwidth (torch copy_ "
                                             "of 2 x 32 MiB, graph-replayed, read + write bytes)",
                                "fetched_bytes_per_ray": round(fetched_per_ray, 2),
                                "nodes_per_ray": round(steps_count["node_steps"] / args.rays, 4),
                                "triangles_per_ray": round(steps_count["triangle_steps"] / args.rays, 4),
                                "bytes": "80 B per 8-wide node visited + 48 B per triangle tested, "
                                         "counted by spb_cast_stats_device over the same rays"}},
            "id_parity": id_parity,
            "any_hit_mrays_s": round(world * any_hit_mrays, 3),
            "render": render,
            "e2e": e2e,
            "cpu_baseline": cpu_baseline,
            "gpu_launches": args.steps,
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))

    tree.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
